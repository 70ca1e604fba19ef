// gfc_serve.cu -- request loop with continuous batching.
//
// Requests (a lattice to gauge-fix: uploaded links or the seeded synthetic
// construction) queue on the host.  Each step admits queued requests, in arrival
// order with first fit, as long as a batch slot and device memory are free; runs one
// round of the batch engine (all admitted lattices advance together, each timeslice
// retiring on its own e2); and finalises the lattices whose timeslices have all
// retired.  Their G stays resident until fetched, then the slot and its memory are
// released for the next request.  Lattices therefore join and leave while others
// are on the GPU, and a lattice's result does not depend on what it shares the GPU
// with (rounds are aligned and every decision is per timeslice).
#include <chrono>
#include <deque>
#include <map>
#include <vector>

#include "gfc.h"
#include "gfc_ctx.h"

namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Request {
    int64_t id;
    int ns, nt, precision;
    int synth;               // 1: seeded synthetic links built on the device
    uint64_t seed;
    double scale;
    std::vector<char> raw;   // uploaded links (copied at submit), elem_bytes / byteswap below
    int elem_bytes, byteswap;
    double t_submit, t_admit = 0, t_done = 0;
    int slot = -1;
    int state = 0;           // 0 queued, 1 running, 2 done (G resident), 3 fetched
    gfc_report report{};
};

}  // namespace

struct gfc_server {
    gfc_batch *b = nullptr;
    int device = 0;
    int64_t next_id = 1;
    std::deque<int64_t> queue;
    std::map<int64_t, Request> req;
    std::map<int, int64_t> slot_req;
    size_t max_sites = 0;
    long long steps = 0;
};

using namespace gfc;

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
    *out = s;
    return GFC_OK;
}

extern "C" int gfc_server_destroy(gfc_server *s) {
    if (!s) return GFC_ERR_ARG;
    gfc_batch_destroy(s->b);
    delete s;
    return GFC_OK;
}

extern "C" size_t gfc_server_capacity_sites(const gfc_server *s) { return s ? s->max_sites : 0; }

// Queue a request.  links == NULL: the synthetic configuration (seed, scale) is
// built on the device at admission; otherwise the raw reference-layout bytes are
// copied now and uploaded at admission.
extern "C" int gfc_server_submit(gfc_server *s, int ns, int nt, const void *links, int elem_bytes, int byteswap,
                                 uint64_t seed, double scale, int precision, int64_t *id) {
    if (!s || !id || ns <= 0 || nt <= 0 || (ns & 1)) return GFC_ERR_ARG;
    const size_t V = (size_t)ns * ns * ns * nt;
    if (V > s->max_sites) {
        set_error("request of %zu sites exceeds the server capacity of %zu sites", V, s->max_sites);
        return GFC_ERR_BUSY;
    }
    Request r;
    r.id = s->next_id++;
    r.ns = ns;
    r.nt = nt;
    r.precision = precision;
    r.synth = links == nullptr;
    r.seed = seed;
    r.scale = scale;
    r.elem_bytes = elem_bytes;
    r.byteswap = byteswap;
    if (links) {
        if (elem_bytes != 8 && elem_bytes != 4) return GFC_ERR_ARG;
        r.raw.assign((const char *)links, (const char *)links + V * 4 * 18 * elem_bytes);
    }
    r.t_submit = now_s();
    *id = r.id;
    s->queue.push_back(r.id);
    s->req.emplace(r.id, std::move(r));
    return GFC_OK;
}

// Admit what fits, run one round, finalise finished lattices.  *running /
// *queued report the state after the step.
extern "C" int gfc_server_step(gfc_server *s, const gfc_params *p, const gfc_options *o, int *running,
                               int *queued) {
    if (!s || !p) return GFC_ERR_ARG;
    // admission: arrival order, first fit
    for (auto it = s->queue.begin(); it != s->queue.end();) {
        Request &r = s->req[*it];
        int slot = -1;
        int rc = gfc_batch_add(s->b, r.ns, r.nt, &slot);
        if (rc == GFC_ERR_BUSY || rc == GFC_ERR_NOMEM) {
            ++it;   // does not fit yet; a later, smaller request may
            continue;
        }
        if (rc) return rc;
        rc = r.synth ? gfc_batch_synth(s->b, slot, r.seed, r.scale)
                     : gfc_batch_upload(s->b, slot, r.raw.data(), r.elem_bytes, r.byteswap);
        if (!rc) rc = gfc_batch_activate(s->b, slot, r.precision);
        if (rc) return rc;
        std::vector<char>().swap(r.raw);
        r.slot = slot;
        r.state = 1;
        r.t_admit = now_s();
        s->slot_req[slot] = r.id;
        it = s->queue.erase(it);
    }
    int active = 0;
    if (!s->slot_req.empty()) {
        int rc = gfc_batch_round(s->b, p, o, &active);
        if (rc) return rc;
        s->steps++;
    }
    int nrun = 0;
    for (auto &kv : s->slot_req) {
        Request &r = s->req[kv.second];
        if (r.state != 1) continue;
        int done = 0;
        gfc_batch_slot_done(s->b, kv.first, &done);
        if (done) {
            int rc = gfc_batch_finalize(s->b, kv.first, &r.report);
            if (rc) return rc;
            r.t_done = now_s();
            r.state = 2;
        } else {
            nrun++;
        }
    }
    if (running) *running = nrun;
    if (queued) *queued = (int)s->queue.size();
    return GFC_OK;
}

// state: 0 queued, 1 running, 2 done (G resident), 3 fetched.  Times in seconds
// since submit: admit, done.  report filled once done.
extern "C" int gfc_server_poll(gfc_server *s, int64_t id, int *state, double *t_admit, double *t_done,
                               gfc_report *report) {
    if (!s) return GFC_ERR_ARG;
    auto it = s->req.find(id);
    if (it == s->req.end()) return GFC_ERR_ARG;
    const Request &r = it->second;
    if (state) *state = r.state;
    if (t_admit) *t_admit = r.state >= 1 ? r.t_admit - r.t_submit : -1.0;
    if (t_done) *t_done = r.state >= 2 ? r.t_done - r.t_submit : -1.0;
    if (report && r.state >= 2) *report = r.report;
    return GFC_OK;
}

// Copy G of a finished request to host memory (elem_bytes 8 or 4) and, with
// release != 0, free its slot and device memory.  gt may be NULL to only release.
extern "C" int gfc_server_fetch(gfc_server *s, int64_t id, void *gt, int elem_bytes, int release) {
    if (!s) return GFC_ERR_ARG;
    auto it = s->req.find(id);
    if (it == s->req.end() || it->second.state != 2) return GFC_ERR_STATE;
    Request &r = it->second;
    if (gt) {
        int rc = gfc_batch_download_gt(s->b, r.slot, gt, elem_bytes, 0);
        if (rc) return rc;
    }
    if (release) {
        int rc = gfc_batch_remove(s->b, r.slot);
        if (rc) return rc;
        s->slot_req.erase(r.slot);
        r.slot = -1;
        r.state = 3;
    }
    return GFC_OK;
}

extern "C" gfc_batch *gfc_server_batch(gfc_server *s) { return s ? s->b : nullptr; }
