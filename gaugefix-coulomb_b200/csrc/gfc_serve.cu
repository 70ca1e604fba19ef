// gfc_serve.cu -- request loop with continuous batching.
//
// Requests (a lattice to gauge-fix: uploaded links or the seeded synthetic
// construction) queue on the host.  Each step releases the device memory of
// requests whose results have reached the host, admits queued requests in arrival
// order with first fit while a batch slot and device memory are free, runs one round
// of the batch engine (all admitted lattices advance together, each timeslice
// retiring on its own e2) and finalises the lattices whose timeslices have all
// retired.  A result thread copies each finished G to host memory on its own
// stream while the next rounds run, so the copy does not stall the device.
// Lattices therefore join and leave while others are on the GPU, and a lattice's
// result does not depend on what it shares the GPU with (rounds are aligned and
// every decision is per timeslice).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "gfc.h"
#include "gfc_ctx.h"

namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

enum { REQ_QUEUED = 0, REQ_RUNNING = 1, REQ_DONE = 2, REQ_FETCHED = 3 };

struct Request {
    int64_t id = 0;
    int ns = 0, nt = 0, precision = 0;
    int synth = 0;           // 1: seeded synthetic links built on the device at admission
    uint64_t seed = 0;
    double scale = 0;
    std::vector<char> raw;   // uploaded links (copied at submit), elem_bytes / byteswap below
    int elem_bytes = 8, byteswap = 0;
    double t_submit = 0, t_admit = 0, t_done = 0;
    int slot = -1;
    int state = REQ_QUEUED;
    int err = 0;             // error of the result copy
    gfc_report report{};
    double *gt = nullptr;    // G in the reference layout once REQ_DONE (from the host pool)
    size_t gt_n = 0;         // doubles
};

// Host buffers for results.  Page-locked buffers are kept and reused (a copy into
// them runs at the link's speed, and pinning is paid once, not per request); past
// `cap` bytes of pinned memory a plain allocation is used instead.  take / give /
// adopt run under the server's lock; allocate runs outside it (pinning is slow).
struct HostPool {
    struct Buf {
        void *p;
        size_t bytes;
        bool pinned;
    };
    std::multimap<size_t, Buf> idle;   // by size
    std::map<void *, Buf> out;         // handed to a request
    size_t pinned_bytes = 0, cap = (size_t)32 << 30;

    // an idle buffer that fits without wasting more than half of it, or null;
    // *pin says whether a new buffer may be pinned (its bytes are then counted)
    void *take(size_t bytes, bool *pin) {
        auto it = idle.lower_bound(bytes);
        if (it != idle.end() && it->first <= 2 * bytes) {
            Buf b = it->second;
            idle.erase(it);
            out[b.p] = b;
            return b.p;
        }
        *pin = pinned_bytes + bytes <= cap;
        if (*pin) pinned_bytes += bytes;
        return nullptr;
    }
    static void *allocate(size_t bytes, bool *pin) {
        void *p = nullptr;
        if (*pin && cudaHostAlloc(&p, bytes, cudaHostAllocDefault) == cudaSuccess) return p;
        cudaGetLastError();
        *pin = false;
        return malloc(bytes);
    }
    void adopt(void *p, size_t bytes, bool pinned_asked, bool pinned) {
        if (pinned_asked && !pinned) pinned_bytes -= bytes;
        if (p) out[p] = Buf{p, bytes, pinned};
    }
    void give(void *p) {
        auto it = out.find(p);
        if (it == out.end()) return;
        Buf b = it->second;
        out.erase(it);
        if (b.pinned)
            idle.emplace(b.bytes, b);
        else
            free(b.p);
    }
    void clear() {
        for (auto &kv : out) kv.second.pinned ? (void)cudaFreeHost(kv.second.p) : free(kv.second.p);
        for (auto &kv : idle) cudaFreeHost(kv.second.p);
        out.clear();
        idle.clear();
        pinned_bytes = 0;
    }
};

// a result buffer from the pool; call without holding the lock
void *pool_get(std::mutex &mu, HostPool &pool, size_t bytes) {
    bool pin = false;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (void *p = pool.take(bytes, &pin)) return p;
    }
    const bool asked = pin;
    void *p = HostPool::allocate(bytes, &pin);
    std::lock_guard<std::mutex> lk(mu);
    pool.adopt(p, bytes, asked, pin);
    return p;
}

struct Job {
    int64_t id;
    int slot;
    size_t sites;
};

}  // namespace

struct gfc_server {
    gfc_batch *b = nullptr;
    int device = 0;
    int64_t next_id = 1;
    size_t max_sites = 0;
    long long steps = 0;
    double sec[4] = {0, 0, 0, 0};     // release, admission, rounds, finalisation
    std::deque<int64_t> queue;        // main thread
    std::map<int, int64_t> slot_req;  // main thread: slots in use (sweeping or copying out)
    int runnable = 0;                 // main thread: slots still sweeping
    int policy = GFC_SERVE_ALL;       // main thread: which admitted requests sweep each round
    size_t work_sites = 0;            //   GFC_SERVE_SMALLEST_FIRST: sites swept together
    std::map<int, int> held;          // main thread: slot -> held by the policy
    // shared with the result thread (under mu)
    std::mutex mu;
    std::condition_variable cv;
    std::map<int64_t, Request> req;   // node-based: references stay valid
    std::deque<Job> jobs;
    std::vector<int> released;        // slots whose G is on the host
    bool stop = false;
    cudaStream_t io = nullptr;
    std::thread worker;
    HostPool host;                    // under mu
};

using namespace gfc;

static void result_thread(gfc_server *s) {
    cudaSetDevice(s->device);
    for (;;) {
        Job j;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv.wait(lk, [s] { return s->stop || !s->jobs.empty(); });
            if (s->jobs.empty()) return;
            j = s->jobs.front();
            s->jobs.pop_front();
        }
        const size_t n = j.sites * 18;
        double *g = (double *)pool_get(s->mu, s->host, n * sizeof(double));
        int rc = GFC_ERR_NOMEM;
        if (g) rc = batch_download_gt_on(s->b, j.slot, g, 8, 0, s->io);
        std::lock_guard<std::mutex> lk(s->mu);
        Request &r = s->req[j.id];
        r.gt = g;
        r.gt_n = g ? n : 0;
        r.err = rc;
        r.t_done = now_s();
        r.state = REQ_DONE;
        s->released.push_back(j.slot);
        s->cv.notify_all();
    }
}

// max_sites: capacity in lattice sites; 0 = as many as `mem_fraction` of the free
// device memory holds (about 1.3 kB per site resident).
extern "C" int gfc_server_create(int device, size_t max_sites, double mem_fraction, int max_slots, int max_nt,
                                 gfc_server **out) {
    if (!out || max_slots <= 0 || max_nt <= 0) return GFC_ERR_ARG;
    *out = nullptr;
    GFC_CHECK(cudaSetDevice(device));
    if (max_sites == 0) {
        size_t fr = 0, tot = 0;
        GFC_CHECK(cudaMemGetInfo(&fr, &tot));
        const double per_site = (double)gfc_batch_slot_bytes(64, 128) / (64.0 * 64 * 64 * 128);
        max_sites = (size_t)((double)fr * (mem_fraction > 0 && mem_fraction < 1 ? mem_fraction : 0.85) / per_site);
    }
    gfc_server *s = new gfc_server();
    s->device = device;
    s->max_sites = max_sites;
    int rc = gfc_batch_create(device, max_sites, max_slots, max_nt, &s->b);
    if (rc) {
        delete s;
        return rc;
    }
    // the capacity is mapped now: admissions then only carve slots out of it
    rc = batch_warm_pool(s->b, (size_t)((double)max_sites * (double)gfc_batch_slot_bytes(64, 128) /
                                        (64.0 * 64 * 64 * 128)));
    if (rc) {
        gfc_batch_destroy(s->b);
        delete s;
        return rc;
    }
    cudaError_t e = cudaStreamCreateWithFlags(&s->io, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        gfc_batch_destroy(s->b);
        delete s;
        return cuda_fail(e, "cudaStreamCreateWithFlags");
    }
    s->worker = std::thread(result_thread, s);
    *out = s;
    return GFC_OK;
}

extern "C" int gfc_server_destroy(gfc_server *s) {
    if (!s) return GFC_ERR_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();   // finishes the copies already queued
    s->host.clear();
    gfc_batch_destroy(s->b);
    cudaStreamDestroy(s->io);
    delete s;
    return GFC_OK;
}

extern "C" size_t gfc_server_capacity_sites(const gfc_server *s) { return s ? s->max_sites : 0; }

// Queue a request.  links == NULL: the synthetic configuration (seed, scale) is
// built on the device at admission; otherwise the raw reference-layout bytes are
// copied now and uploaded at admission.
extern "C" int gfc_server_submit(gfc_server *s, int ns, int nt, const void *links, int elem_bytes, int byteswap,
                                 uint64_t seed, double scale, int precision, int64_t *id) {
    if (!s || !id || ns <= 0 || nt <= 0) return GFC_ERR_ARG;
    if (links && elem_bytes != 8 && elem_bytes != 4) return GFC_ERR_ARG;
    const size_t V = (size_t)ns * ns * ns * nt;
    if (V > s->max_sites) {
        set_error("request of %zu sites exceeds the server capacity of %zu sites", V, s->max_sites);
        return GFC_ERR_BUSY;
    }
    Request r;
    r.ns = ns;
    r.nt = nt;
    r.precision = precision;
    r.synth = links == nullptr;
    r.seed = seed;
    r.scale = scale;
    r.elem_bytes = elem_bytes;
    r.byteswap = byteswap;
    if (links) r.raw.assign((const char *)links, (const char *)links + V * 4 * 18 * elem_bytes);
    r.t_submit = now_s();
    std::lock_guard<std::mutex> lk(s->mu);
    r.id = s->next_id++;
    *id = r.id;
    s->queue.push_back(r.id);
    s->req.emplace(r.id, std::move(r));
    return GFC_OK;
}

// Release, admit, run one round, finalise.  *running / *queued: requests on the
// device (including those whose result is being copied) and waiting.
extern "C" int gfc_server_step(gfc_server *s, const gfc_params *p, const gfc_options *o, int *running,
                               int *queued) {
    if (!s || !p) return GFC_ERR_ARG;
    double t0 = now_s();
    // results on the host: give their device memory back.  With nothing left to
    // sweep but copies in flight, wait (briefly) for one instead of spinning.
    std::vector<int> rel;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        if (s->released.empty() && s->runnable == 0 && !s->slot_req.empty())
            s->cv.wait_for(lk, std::chrono::milliseconds(20), [s] { return !s->released.empty(); });
        rel.swap(s->released);
    }
    for (int slot : rel) {
        int rc = gfc_batch_remove(s->b, slot);
        if (rc) return rc;
        s->slot_req.erase(slot);
        s->held.erase(slot);
    }
    double t1 = now_s();
    s->sec[0] += t1 - t0;
    // admission: arrival order, first fit
    for (auto it = s->queue.begin(); it != s->queue.end();) {
        Request *r;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            r = &s->req[*it];
        }
        int slot = -1;
        int rc = gfc_batch_add(s->b, r->ns, r->nt, &slot);
        if (rc == GFC_ERR_BUSY || rc == GFC_ERR_NOMEM) {
            ++it;   // does not fit yet; a later, smaller request may
            continue;
        }
        if (rc) return rc;
        rc = r->synth ? gfc_batch_synth(s->b, slot, r->seed, r->scale)
                      : gfc_batch_upload(s->b, slot, r->raw.data(), r->elem_bytes, r->byteswap);
        if (!rc) rc = gfc_batch_activate(s->b, slot, r->precision);
        if (rc) return rc;
        std::vector<char>().swap(r->raw);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            r->slot = slot;
            r->state = REQ_RUNNING;
            r->t_admit = now_s();
        }
        s->slot_req[slot] = r->id;
        s->runnable++;
        it = s->queue.erase(it);
    }
    // which admitted requests sweep in this round
    if (s->policy == GFC_SERVE_SMALLEST_FIRST) {
        std::vector<std::pair<size_t, int64_t>> run;   // (sites, id) of requests still sweeping
        {
            std::lock_guard<std::mutex> lk(s->mu);
            for (auto &kv : s->slot_req) {
                const Request &r = s->req[kv.second];
                if (r.state == REQ_RUNNING && r.slot >= 0)
                    run.push_back({(size_t)r.ns * r.ns * r.ns * r.nt, r.id});
            }
        }
        std::sort(run.begin(), run.end());
        size_t cum = 0;
        for (auto &e : run) {
            int slot;
            {
                std::lock_guard<std::mutex> lk(s->mu);
                slot = s->req[e.second].slot;
            }
            const int hold = cum > 0 && cum + e.first > s->work_sites;
            if (!hold) cum += e.first;
            if (s->held[slot] != hold) {
                int rc = gfc_batch_hold(s->b, slot, hold);
                if (rc) return rc;
                s->held[slot] = hold;
            }
        }
    }
    double t2 = now_s();
    s->sec[1] += t2 - t1;
    int active = 0;
    if (s->runnable > 0) {
        int rc = gfc_batch_round(s->b, p, o, &active);
        if (rc) return rc;
        s->steps++;
    }
    double t3 = now_s();
    s->sec[2] += t3 - t2;
    // finished lattices: finalise here, copy G on the result thread
    int nfin = 0;
    for (auto &kv : s->slot_req) {
        Request *r;
        bool mine;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            r = &s->req[kv.second];
            mine = r->state == REQ_RUNNING && r->slot >= 0;   // not yet handed to the result thread
        }
        if (!mine) continue;
        int done = 0;
        gfc_batch_slot_done(s->b, kv.first, &done);
        if (!done) continue;
        gfc_report rep{};
        int rc = gfc_batch_finalize(s->b, kv.first, &rep);
        if (rc) return rc;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            r->report = rep;
            r->slot = -1;   // handed to the result thread
            s->jobs.push_back(Job{r->id, kv.first, (size_t)r->ns * r->ns * r->ns * r->nt});
        }
        s->runnable--;
        nfin++;
    }
    if (nfin) s->cv.notify_all();
    s->sec[3] += now_s() - t3;
    if (running) *running = (int)s->slot_req.size();
    if (queued) *queued = (int)s->queue.size();
    return GFC_OK;
}

// state: 0 queued, 1 running (or its G on the way to the host), 2 done (G on the
// host, device memory released at the next step), 3 fetched.  Times in seconds
// after submit: admission and result on the host.  report filled once done.
extern "C" int gfc_server_poll(gfc_server *s, int64_t id, int *state, double *t_admit, double *t_done,
                               gfc_report *report) {
    if (!s) return GFC_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->req.find(id);
    if (it == s->req.end()) return GFC_ERR_ARG;
    const Request &r = it->second;
    if (state) *state = r.state;
    if (t_admit) *t_admit = r.state >= REQ_RUNNING ? r.t_admit - r.t_submit : -1.0;
    if (t_done) *t_done = r.state >= REQ_DONE ? r.t_done - r.t_submit : -1.0;
    if (report && r.state >= REQ_DONE) *report = r.report;
    return GFC_OK;
}

// Copy G of a finished request (reference layout, elem_bytes 8 or 4) to `gt`;
// with release != 0 the host copy is dropped.  gt may be NULL to only release.
extern "C" int gfc_server_fetch(gfc_server *s, int64_t id, void *gt, int elem_bytes, int release) {
    if (!s || (gt && elem_bytes != 8 && elem_bytes != 4)) return GFC_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->req.find(id);
    if (it == s->req.end() || it->second.state != REQ_DONE) return GFC_ERR_STATE;
    Request &r = it->second;
    if (r.err) return r.err;
    if (gt) {
        if (elem_bytes == 8) {
            memcpy(gt, r.gt, r.gt_n * sizeof(double));
        } else {
            float *f = (float *)gt;
            for (size_t k = 0; k < r.gt_n; k++) f[k] = (float)r.gt[k];
        }
    }
    if (release) {
        s->host.give(r.gt);
        r.gt = nullptr;
        r.gt_n = 0;
        r.state = REQ_FETCHED;
    }
    return GFC_OK;
}

extern "C" int gfc_server_result(gfc_server *s, int64_t id, const double **gt, size_t *count) {
    if (!s || !gt || !count) return GFC_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->req.find(id);
    if (it == s->req.end() || it->second.state != REQ_DONE) return GFC_ERR_STATE;
    if (it->second.err) return it->second.err;
    *gt = it->second.gt;
    *count = it->second.gt_n;
    return GFC_OK;
}

// Pin `bytes` of host memory for results now (buffers of the given size), so the
// first large results do not wait for page locking.
extern "C" int gfc_server_reserve_host(gfc_server *s, size_t buffer_bytes, int count) {
    if (!s || count < 0) return GFC_ERR_ARG;
    std::vector<void *> got;
    for (int k = 0; k < count; k++) {
        void *p = pool_get(s->mu, s->host, buffer_bytes);
        if (!p) break;
        got.push_back(p);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    for (void *p : got) s->host.give(p);
    return (int)got.size() == count ? GFC_OK : GFC_ERR_NOMEM;
}

// Scheduling of admitted requests.  GFC_SERVE_ALL: every admitted request sweeps in
// every round (they share the GPU).  GFC_SERVE_SMALLEST_FIRST: the requests still
// sweeping are taken smallest first until work_sites sites are sweeping (at least
// one); the others stay resident and wait.  Admission is by free memory either way.
extern "C" int gfc_server_set_policy(gfc_server *s, int policy, size_t work_sites) {
    if (!s || (policy != GFC_SERVE_ALL && policy != GFC_SERVE_SMALLEST_FIRST)) return GFC_ERR_ARG;
    if (policy == GFC_SERVE_ALL)
        for (auto &kv : s->held)
            if (kv.second) {
                int rc = gfc_batch_hold(s->b, kv.first, 0);
                if (rc) return rc;
                kv.second = 0;
            }
    s->policy = policy;
    s->work_sites = work_sites;
    return GFC_OK;
}

// Host seconds spent in the four phases of gfc_server_step (release, admission,
// rounds, finalisation) and the number of rounds run.
extern "C" int gfc_server_stats(const gfc_server *s, double *seconds4, long long *rounds) {
    if (!s) return GFC_ERR_ARG;
    if (seconds4)
        for (int k = 0; k < 4; k++) seconds4[k] = s->sec[k];
    if (rounds) *rounds = s->steps;
    return GFC_OK;
}

extern "C" gfc_batch *gfc_server_batch(gfc_server *s) { return s ? s->b : nullptr; }
