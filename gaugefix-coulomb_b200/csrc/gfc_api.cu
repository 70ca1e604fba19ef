// gfc_api.cu -- C ABI: device contexts, chunked host <-> device transfers, the
// gauge-fixing driver loop, observables.
//
// The driver loop reproduces gaugefixOverrelaxation (gauge_fixing.c:713-826):
// G = 1, proxy, the check schedule of whenNextConvergenceCheckQ
// (gauge_fixing.c:248-285), the stall test |dres|/res < 10E-16, max_sweeps and the
// reunitarisation every sweeps_to_reunitarization half-sweeps, then a final
// reunitarisation.  Half-sweeps are queued asynchronously; the host waits only at
// scheduled checks (one double comes back).
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>

#include "gfc.h"
#include "gfc_ctx.h"
#include "gfc_fast.h"

namespace gfc {

static thread_local char g_err[512];

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

int cuda_fail(cudaError_t e, const char *what) {
    set_error("%s: %s", what, cudaGetErrorString(e));
    return GFC_ERR_CUDA;
}

}  // namespace gfc

using namespace gfc;

extern "C" const char *gfc_last_error(void) { return g_err; }

// ------------------------------------------------------------------ contexts --
static void ctx_free(gfc_ctx *c) {
    if (!c) return;
    cudaSetDevice(c->dev);
    cudaFree(c->u);
    cudaFree(c->g);
    cudaFree(c->ut);
    cudaFree(c->u0);
    cudaFree(c->backup);
    cudaFree(c->u64r);
    cudaFree(c->g64r);
    cudaFree(c->u32);
    cudaFree(c->g32);
    cudaFree(c->part);
    cudaFree(c->dres);
    cudaFree(c->dstatus);
    cudaFree(c->e2_slice);
    cudaFree(c->e2_hist);
    cudaFree(c->tickets);
    cudaFree(c->ring);
    for (int k = 0; k < 2; k++) {
        cudaFree(c->dstage[k]);
        cudaFreeHost(c->hstage[k]);
        if (c->ev_copy[k]) cudaEventDestroy(c->ev_copy[k]);
        if (c->ev_used[k]) cudaEventDestroy(c->ev_used[k]);
    }
    cudaFreeHost(c->hres);
    if (c->ev_a) cudaEventDestroy(c->ev_a);
    if (c->ev_b) cudaEventDestroy(c->ev_b);
    if (c->ev_c) cudaEventDestroy(c->ev_c);
    if (c->ev_d) cudaEventDestroy(c->ev_d);
    if (c->s) cudaStreamDestroy(c->s);
    if (c->sc) cudaStreamDestroy(c->sc);
    delete c;
}

extern "C" int gfc_ctx_create(int ns, int nt, int device, int flags, gfc_ctx **out) {
    if (!out) return GFC_ERR_ARG;
    *out = nullptr;
    if (ns <= 0 || nt <= 0) {
        set_error("bad lattice extents ns=%d nt=%d", ns, nt);
        return GFC_ERR_GEOMETRY;
    }
    uint64_t V = (uint64_t)ns * ns * ns * nt;
    if (V * 4 >= (1ull << 31)) {
        set_error("lattice %d^3x%d too large for 32-bit site indices", ns, nt);
        return GFC_ERR_GEOMETRY;
    }
    gfc_ctx *c = new gfc_ctx();
    c->dev = device;
    c->lat = make_lat(ns, nt);
    const Lat &l = c->lat;
    int rc = GFC_OK;
#define TRY(call)                                 \
    do {                                          \
        cudaError_t _e = (call);                  \
        if (_e != cudaSuccess) {                  \
            rc = cuda_fail(_e, #call);            \
            goto fail;                            \
        }                                         \
    } while (0)
    {
        TRY(cudaSetDevice(device));
        TRY(cudaStreamCreateWithFlags(&c->s, cudaStreamNonBlocking));
        TRY(cudaStreamCreateWithFlags(&c->sc, cudaStreamNonBlocking));
        size_t mat = (size_t)l.npar * l.vh * 9;  // double2 per full field
        TRY(cudaMalloc(&c->u, 3 * mat * sizeof(double2)));
        TRY(cudaMalloc(&c->g, mat * sizeof(double2)));
        TRY(cudaMalloc(&c->ut, mat * sizeof(double2)));
        if (flags & GFC_CTX_MIXED) {
            TRY(cudaMalloc(&c->u0, 3 * mat * sizeof(double2)));
            TRY(cudaMalloc(&c->u32, 3 * (size_t)l.npar * l.vh * 6 * sizeof(float2)));
            TRY(cudaMalloc(&c->g32, (size_t)l.npar * l.vh * 6 * sizeof(float2)));
        }
        int nbx = obs_blocks_per_slice(l);
        c->part_n = (size_t)nt * nbx * 4;
        TRY(cudaMalloc(&c->part, c->part_n * sizeof(double)));
        TRY(cudaMalloc(&c->dres, 32 * sizeof(double)));
        TRY(cudaMalloc(&c->dstatus, sizeof(unsigned)));
        TRY(cudaMemset(c->dstatus, 0, sizeof(unsigned)));
        TRY(cudaMalloc(&c->e2_slice, (size_t)nt * 2 * sizeof(double)));
        TRY(cudaMallocHost(&c->hres, 32 * sizeof(double)));
        TRY(cudaEventCreate(&c->ev_a));
        TRY(cudaEventCreate(&c->ev_b));
        TRY(cudaEventCreate(&c->ev_c));
        TRY(cudaEventCreate(&c->ev_d));
        TRY(cudaMalloc(&c->tickets, (size_t)(nt + 2) * sizeof(unsigned)));
        TRY(cudaMemset(c->tickets, 0, (size_t)(nt + 2) * sizeof(unsigned)));
        // staging: a whole number of timeslices of FP64 links, at most ~64 MB
        size_t slice_bytes = (size_t)l.vs * 4 * 144;
        size_t nts = std::max<size_t>(1, ((size_t)64 << 20) / slice_bytes);
        if (nts > (size_t)nt) nts = nt;
        c->stage_bytes = nts * slice_bytes;
        for (int k = 0; k < 2; k++) {
            TRY(cudaMalloc(&c->dstage[k], c->stage_bytes));
            TRY(cudaMallocHost(&c->hstage[k], c->stage_bytes));
            TRY(cudaEventCreateWithFlags(&c->ev_copy[k], cudaEventDisableTiming));
            TRY(cudaEventCreateWithFlags(&c->ev_used[k], cudaEventDisableTiming));
        }
    }
#undef TRY
    *out = c;
    return GFC_OK;
fail:
    ctx_free(c);
    return rc;
}

extern "C" int gfc_ctx_destroy(gfc_ctx *c) {
    if (!c) return GFC_ERR_ARG;
    cudaSetDevice(c->dev);
    cudaStreamSynchronize(c->s);
    cudaStreamSynchronize(c->sc);
    ctx_free(c);
    return GFC_OK;
}

extern "C" void *gfc_host_alloc(size_t bytes) {
    void *p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

extern "C" void gfc_host_free(void *p) {
    if (p) cudaFreeHost(p);
}

extern "C" long long gfc_ctx_kernel_launches(const gfc_ctx *c) { return c ? c->launches : -1; }

extern "C" void *gfc_ctx_stream(gfc_ctx *c) { return c ? (void *)c->s : nullptr; }

// ------------------------------------------------------- chunked transfers --
static int is_pinned(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return a.type == cudaMemoryTypeHost;
}

// Host -> device of a raw per-timeslice-ordered array; calls fn(dptr, t0, nts)
// on the compute stream for each chunk once it is on the device.
template <typename F>
static int upload_chunked(gfc_ctx *c, const void *host, size_t bytes_per_slice, F fn) {
    const Lat &l = c->lat;
    uint32_t per = (uint32_t)std::max<size_t>(1, c->stage_bytes / bytes_per_slice);
    const int pinned = is_pinned(host);
    int k = 0;
    for (uint32_t t0 = 0; t0 < (uint32_t)l.nt; t0 += per, k ^= 1) {
        uint32_t nts = std::min<uint32_t>(per, l.nt - t0);
        size_t bytes = (size_t)nts * bytes_per_slice;
        const char *src = (const char *)host + (size_t)t0 * bytes_per_slice;
        // the staging buffer k must be free (its previous transform done)
        GFC_CHECK(cudaStreamWaitEvent(c->sc, c->ev_used[k], 0));
        if (pinned) {
            GFC_CHECK(cudaMemcpyAsync(c->dstage[k], src, bytes, cudaMemcpyHostToDevice, c->sc));
        } else {
            GFC_CHECK(cudaEventSynchronize(c->ev_copy[k]));  // host staging k reusable
            memcpy(c->hstage[k], src, bytes);
            GFC_CHECK(cudaMemcpyAsync(c->dstage[k], c->hstage[k], bytes, cudaMemcpyHostToDevice, c->sc));
        }
        GFC_CHECK(cudaEventRecord(c->ev_copy[k], c->sc));
        GFC_CHECK(cudaStreamWaitEvent(c->s, c->ev_copy[k], 0));
        fn(c->dstage[k], t0, nts);
        c->launches++;
        GFC_CHECK(cudaEventRecord(c->ev_used[k], c->s));
    }
    GFC_CHECK(cudaGetLastError());
    return GFC_OK;
}

template <typename F>
static int download_chunked(gfc_ctx *c, void *host, size_t bytes_per_slice, F fn, int wait = 1) {
    const Lat &l = c->lat;
    uint32_t per = (uint32_t)std::max<size_t>(1, c->stage_bytes / bytes_per_slice);
    const int pinned = is_pinned(host);
    if (!wait && !pinned) return GFC_ERR_ARG;   // an unfinished copy must land in page-locked memory
    int k = 0;
    uint32_t pend_t0[2] = {0, 0}, pend_n[2] = {0, 0};
    int pend[2] = {0, 0};
    for (uint32_t t0 = 0; t0 < (uint32_t)l.nt; t0 += per, k ^= 1) {
        uint32_t nts = std::min<uint32_t>(per, l.nt - t0);
        size_t bytes = (size_t)nts * bytes_per_slice;
        // staging k must have been copied out
        GFC_CHECK(cudaStreamWaitEvent(c->s, c->ev_copy[k], 0));
        if (!pinned && pend[k]) {
            GFC_CHECK(cudaEventSynchronize(c->ev_copy[k]));
            memcpy((char *)host + (size_t)pend_t0[k] * bytes_per_slice, c->hstage[k],
                   (size_t)pend_n[k] * bytes_per_slice);
            pend[k] = 0;
        }
        fn(c->dstage[k], t0, nts);
        c->launches++;
        GFC_CHECK(cudaEventRecord(c->ev_used[k], c->s));
        GFC_CHECK(cudaStreamWaitEvent(c->sc, c->ev_used[k], 0));
        void *dst = pinned ? (char *)host + (size_t)t0 * bytes_per_slice : c->hstage[k];
        GFC_CHECK(cudaMemcpyAsync(dst, c->dstage[k], bytes, cudaMemcpyDeviceToHost, c->sc));
        GFC_CHECK(cudaEventRecord(c->ev_copy[k], c->sc));
        if (!pinned) {
            pend[k] = 1;
            pend_t0[k] = t0;
            pend_n[k] = nts;
        }
    }
    if (!wait) {
        GFC_CHECK(cudaGetLastError());
        return GFC_OK;
    }
    GFC_CHECK(cudaStreamSynchronize(c->sc));
    for (int j = 0; j < 2; j++)
        if (pend[j])
            memcpy((char *)host + (size_t)pend_t0[j] * bytes_per_slice, c->hstage[j],
                   (size_t)pend_n[j] * bytes_per_slice);
    GFC_CHECK(cudaGetLastError());
    return GFC_OK;
}

extern "C" int gfc_ctx_upload_links(gfc_ctx *c, const void *host, int elem_bytes, int byteswap) {
    if (!c || !host || (elem_bytes != 8 && elem_bytes != 4)) return GFC_ERR_ARG;
    GFC_CHECK(cudaSetDevice(c->dev));
    const Lat l = c->lat;
    size_t per_slice = (size_t)l.vs * 4 * 18 * elem_bytes;
    int rc = upload_chunked(c, host, per_slice, [&](void *d, uint32_t t0, uint32_t nts) {
        launch_load_links(d, elem_bytes, byteswap, l, t0, nts, c->u, c->ut, c->s);
    });
    if (rc == GFC_OK) c->has_links = 1;
    return rc;
}

// loadConfig + reunitarizeField (gauge_fix_coulomb.c:123-131) in one pass: the
// same links, bit for bit, as gfc_ctx_upload_links followed by gfc_ctx_reunitarize.
extern "C" int gfc_ctx_upload_links_reunit(gfc_ctx *c, const void *host, int elem_bytes, int byteswap) {
    if (!c || !host || (elem_bytes != 8 && elem_bytes != 4)) return GFC_ERR_ARG;
    GFC_CHECK(cudaSetDevice(c->dev));
    const Lat l = c->lat;
    size_t per_slice = (size_t)l.vs * 4 * 18 * elem_bytes;
    int rc = upload_chunked(c, host, per_slice, [&](void *d, uint32_t t0, uint32_t nts) {
        launch_load_links(d, elem_bytes, byteswap, l, t0, nts, c->u, c->ut, c->s, 1, c->dstatus);
    });
    if (rc == GFC_OK) c->has_links = 1;
    return rc;
}

extern "C" int gfc_ctx_upload_gt(gfc_ctx *c, const void *host, int elem_bytes, int byteswap) {
    if (!c || !host || (elem_bytes != 8 && elem_bytes != 4)) return GFC_ERR_ARG;
    GFC_CHECK(cudaSetDevice(c->dev));
    const Lat l = c->lat;
    size_t per_slice = (size_t)l.vs * 18 * elem_bytes;
    return upload_chunked(c, host, per_slice, [&](void *d, uint32_t t0, uint32_t nts) {
        launch_load_gt(d, elem_bytes, byteswap, l, t0, nts, c->g, c->s);
    });
}

extern "C" int gfc_ctx_download_gt(gfc_ctx *c, void *host, int elem_bytes, int byteswap) {
    if (!c || !host || (elem_bytes != 8 && elem_bytes != 4)) return GFC_ERR_ARG;
    GFC_CHECK(cudaSetDevice(c->dev));
    const Lat l = c->lat;
    size_t per_slice = (size_t)l.vs * 18 * elem_bytes;
    return download_chunked(c, host, per_slice, [&](void *d, uint32_t t0, uint32_t nts) {
        launch_store_gt(c->g, l, t0, nts, elem_bytes, byteswap, d, c->s);
    });
}

// The same as gfc_ctx_download_gt, left in flight on the context's streams: the
// host buffer must be page-locked; gfc_ctx_sync completes it.
extern "C" int gfc_ctx_download_gt_async(gfc_ctx *c, void *host, int elem_bytes, int byteswap) {
    if (!c || !host || (elem_bytes != 8 && elem_bytes != 4)) return GFC_ERR_ARG;
    if (!is_pinned(host)) {
        set_error("gfc_ctx_download_gt_async: the host buffer is not page-locked");
        return GFC_ERR_ARG;
    }
    GFC_CHECK(cudaSetDevice(c->dev));
    const Lat l = c->lat;
    size_t per_slice = (size_t)l.vs * 18 * elem_bytes;
    return download_chunked(
        c, host, per_slice,
        [&](void *d, uint32_t t0, uint32_t nts) { launch_store_gt(c->g, l, t0, nts, elem_bytes, byteswap, d, c->s); },
        0);
}

extern "C" int gfc_ctx_download_links(gfc_ctx *c, void *host, int elem_bytes, int byteswap) {
    if (!c || !host || (elem_bytes != 8 && elem_bytes != 4)) return GFC_ERR_ARG;
    if (!c->has_links) return GFC_ERR_STATE;
    GFC_CHECK(cudaSetDevice(c->dev));
    const Lat l = c->lat;
    size_t per_slice = (size_t)l.vs * 4 * 18 * elem_bytes;
    return download_chunked(c, host, per_slice, [&](void *d, uint32_t t0, uint32_t nts) {
        launch_store_links(c->u, c->ut, l, t0, nts, elem_bytes, byteswap, d, c->s);
    });
}

// ---------------------------------------------------------------- fields --
extern "C" int gfc_ctx_get_link(gfc_ctx *c, size_t site, int mu, double *out18) {
    if (!c || !out18 || mu < 0 || mu > 3 || site >= c->lat.v) return GFC_ERR_ARG;
    if (!c->has_links) return GFC_ERR_STATE;
    GFC_CHECK(cudaSetDevice(c->dev));
    const Lat &l = c->lat;
    Slot s = slot_of(l, (uint32_t)site);
    const double2 *base = mu == 0 ? c->ut + gidx(l, s.par, 0, s.i) : c->u + uidx(l, mu - 1, s.par, 0, s.i);
    for (int k = 0; k < 9; k++)
        GFC_CHECK(cudaMemcpyAsync(out18 + 2 * k, base + (size_t)k * l.vh, sizeof(double2), cudaMemcpyDeviceToHost,
                                  c->s));
    GFC_CHECK(cudaStreamSynchronize(c->s));
    return GFC_OK;
}

static int reunit_spatial_and_g(gfc_ctx *c) {
    const Lat &l = c->lat;
    launch_reunitarize(c->u, l.vh, 3 * l.npar, c->dstatus, c->s);
    launch_reunitarize(c->g, l.vh, l.npar, c->dstatus, c->s);
    c->launches += 2;
    return GFC_OK;
}

extern "C" int gfc_ctx_reunitarize(gfc_ctx *c) {
    if (!c) return GFC_ERR_ARG;
    if (!c->has_links) return GFC_ERR_STATE;
    GFC_CHECK(cudaSetDevice(c->dev));
    const Lat &l = c->lat;
    launch_reunitarize(c->u, l.vh, 3 * l.npar, c->dstatus, c->s);
    launch_reunitarize(c->ut, l.vh, l.npar, c->dstatus, c->s);
    c->launches += 2;
    GFC_CHECK(cudaGetLastError());
    return GFC_OK;
}

// Device-side copy of all links (spatial and temporal), to restart a fix from the
// same configuration without another host transfer.
extern "C" int gfc_ctx_save_links(gfc_ctx *c) {
    if (!c) return GFC_ERR_ARG;
    if (!c->has_links) return GFC_ERR_STATE;
    GFC_CHECK(cudaSetDevice(c->dev));
    const size_t mat = (size_t)c->lat.npar * c->lat.vh * 9 * sizeof(double2);
    if (!c->backup) GFC_CHECK(cudaMalloc(&c->backup, 4 * mat));
    GFC_CHECK(cudaMemcpyAsync(c->backup, c->u, 3 * mat, cudaMemcpyDeviceToDevice, c->s));
    GFC_CHECK(cudaMemcpyAsync((char *)c->backup + 3 * mat, c->ut, mat, cudaMemcpyDeviceToDevice, c->s));
    return GFC_OK;
}

extern "C" int gfc_ctx_restore_links(gfc_ctx *c) {
    if (!c) return GFC_ERR_ARG;
    if (!c->backup) return GFC_ERR_STATE;
    GFC_CHECK(cudaSetDevice(c->dev));
    const size_t mat = (size_t)c->lat.npar * c->lat.vh * 9 * sizeof(double2);
    GFC_CHECK(cudaMemcpyAsync(c->u, c->backup, 3 * mat, cudaMemcpyDeviceToDevice, c->s));
    GFC_CHECK(cudaMemcpyAsync(c->ut, (char *)c->backup + 3 * mat, mat, cudaMemcpyDeviceToDevice, c->s));
    return GFC_OK;
}

extern "C" int gfc_ctx_reunitarize_gt(gfc_ctx *c) {
    if (!c) return GFC_ERR_ARG;
    GFC_CHECK(cudaSetDevice(c->dev));
    launch_reunitarize(c->g, c->lat.vh, c->lat.npar, c->dstatus, c->s);
    c->launches++;
    GFC_CHECK(cudaGetLastError());
    return GFC_OK;
}

extern "C" int gfc_ctx_set_identity_gt(gfc_ctx *c) {
    if (!c) return GFC_ERR_ARG;
    GFC_CHECK(cudaSetDevice(c->dev));
    launch_identity(c->g, c->lat, c->s);
    c->launches += c->lat.npar;
    GFC_CHECK(cudaGetLastError());
    return GFC_OK;
}

// Read and clear the device status word (projection failures, NaN).
extern "C" int gfc_ctx_status(gfc_ctx *c, unsigned *status) {
    if (!c || !status) return GFC_ERR_ARG;
    GFC_CHECK(cudaSetDevice(c->dev));
    unsigned h = 0;
    GFC_CHECK(cudaMemcpyAsync(&h, c->dstatus, sizeof h, cudaMemcpyDeviceToHost, c->s));
    GFC_CHECK(cudaMemsetAsync(c->dstatus, 0, sizeof h, c->s));
    GFC_CHECK(cudaStreamSynchronize(c->s));
    *status = h;
    return GFC_OK;
}

// ------------------------------------------------------------ observables --
static int read_results(gfc_ctx *c, int n) {
    GFC_CHECK(cudaMemcpyAsync(c->hres, c->dres, n * sizeof(double), cudaMemcpyDeviceToHost, c->s));
    GFC_CHECK(cudaStreamSynchronize(c->s));
    return GFC_OK;
}

// e2 (calculate_e2) and theta (calculateTheta) of the current spatial links.
static int obs_e2_theta(gfc_ctx *c, double *e2, double *theta, double *slices) {
    const Lat &l = c->lat;
    launch_obs(c->u, l, c->part, c->dres, c->e2_slice, c->s);
    c->launches += 2;
    GFC_CHECK(cudaGetLastError());
    int rc = read_results(c, 2);
    if (rc) return rc;
    if (e2) *e2 = c->hres[0] / (double)l.v;
    if (theta) *theta = c->hres[1] / (3.0 * (double)l.v);
    if (slices) {
        GFC_CHECK(cudaMemcpy(slices, c->e2_slice, (size_t)l.nt * 2 * sizeof(double), cudaMemcpyDeviceToHost));
        for (int t = 0; t < l.nt; t++) slices[2 * t] /= (double)l.vs;
    }
    return GFC_OK;
}

extern "C" int gfc_ctx_e2(gfc_ctx *c, double *e2, double *theta) {
    if (!c) return GFC_ERR_ARG;
    if (!c->has_links) return GFC_ERR_STATE;
    GFC_CHECK(cudaSetDevice(c->dev));
    return obs_e2_theta(c, e2, theta, nullptr);
}

// per-timeslice e2 (density per slice, normalised by the spatial volume), nt values
extern "C" int gfc_ctx_e2_slices(gfc_ctx *c, double *e2_per_slice) {
    if (!c || !e2_per_slice) return GFC_ERR_ARG;
    if (!c->has_links) return GFC_ERR_STATE;
    GFC_CHECK(cudaSetDevice(c->dev));
    const Lat &l = c->lat;
    double *tmp = (double *)malloc((size_t)l.nt * 2 * sizeof(double));
    if (!tmp) return GFC_ERR_NOMEM;
    int rc = obs_e2_theta(c, nullptr, nullptr, tmp);
    if (rc == GFC_OK)
        for (int t = 0; t < l.nt; t++) e2_per_slice[t] = tmp[2 * t];
    free(tmp);
    return rc;
}

extern "C" int gfc_ctx_functional(gfc_ctx *c, double *F) {
    if (!c || !F) return GFC_ERR_ARG;
    if (!c->has_links) return GFC_ERR_STATE;
    GFC_CHECK(cudaSetDevice(c->dev));
    const Lat &l = c->lat;
    launch_functional(c->u, l, c->part, c->dres, c->s);
    c->launches += 2;
    GFC_CHECK(cudaGetLastError());
    int rc = read_results(c, 1);
    if (rc) return rc;
    *F = c->hres[0] / ((double)l.v * 9.0);
    return GFC_OK;
}

extern "C" int gfc_ctx_plaquette(gfc_ctx *c, double *spatial, double *temporal) {
    if (!c) return GFC_ERR_ARG;
    if (!c->has_links) return GFC_ERR_STATE;
    GFC_CHECK(cudaSetDevice(c->dev));
    const Lat &l = c->lat;
    launch_plaquette(c->u, c->ut, l, c->part, c->dres, c->s);
    c->launches += 2;
    GFC_CHECK(cudaGetLastError());
    int rc = read_results(c, 2);
    if (rc) return rc;
    if (spatial) *spatial = c->hres[0] / (3.0 * (double)l.v);
    if (temporal) *temporal = c->hres[1] / (3.0 * (double)l.v);
    return GFC_OK;
}

// ------------------------------------------------------------ sweeping --
extern "C" int gfc_ctx_halfsweeps(gfc_ctx *c, int first_sweep, int n, float omega_OR, unsigned hits,
                                  int precision) {
    if (!c || n < 0) return GFC_ERR_ARG;
    if (!c->has_links) return GFC_ERR_STATE;
    GFC_CHECK(cudaSetDevice(c->dev));
    const double omega = (double)omega_OR;
    // ns = 1 (one link per direction closing on its site) on the reference-arithmetic
    // kernel whatever the precision: the fast staged forms update that link once
    if (precision == GFC_PREC_FP64_EXACT || c->lat.ns == 1) {
        for (int k = 0; k < n; k++) {
            c->launches += launch_sweep_exact(c->u, c->g, c->lat, first_sweep + k, omega, hits, c->s, c->shape_exact);
        }
    } else if (n > 0) {
        int rc = c->lat.cb ? halfsweeps_fast64(c, first_sweep, n, omega, hits)
                           : halfsweeps_odd_fast(c, first_sweep, n, omega, hits);
        if (rc) return rc;
    }
    GFC_CHECK(cudaGetLastError());
    return GFC_OK;
}

// applyGaugeTransformationU (fields.c:375-435) with the resident G on all links.
extern "C" int gfc_ctx_apply_gt(gfc_ctx *c) {
    if (!c) return GFC_ERR_ARG;
    if (!c->has_links) return GFC_ERR_STATE;
    GFC_CHECK(cudaSetDevice(c->dev));
    launch_apply_gt(c->u, c->ut, c->g, c->lat, 1, c->s);
    c->launches++;
    GFC_CHECK(cudaGetLastError());
    return GFC_OK;
}

extern "C" int gfc_ctx_finalize_temporal(gfc_ctx *c) {
    if (!c) return GFC_ERR_ARG;
    GFC_CHECK(cudaSetDevice(c->dev));
    const Lat &l = c->lat;
    launch_temporal_transform(c->ut, c->g, l, c->s);
    launch_reunitarize(c->ut, l.vh, l.npar, c->dstatus, c->s);
    c->launches += 2;
    GFC_CHECK(cudaGetLastError());
    return GFC_OK;
}

extern "C" int gfc_ctx_sync(gfc_ctx *c) {
    if (!c) return GFC_ERR_ARG;
    GFC_CHECK(cudaSetDevice(c->dev));
    GFC_CHECK(cudaStreamSynchronize(c->s));
    GFC_CHECK(cudaStreamSynchronize(c->sc));   // copies left in flight (gfc_ctx_download_gt_async)
    return GFC_OK;
}

// whenNextConvergenceCheckQ (gauge_fixing.c:248-285)
static int next_check(unsigned sweep, double res, const gfc_params *p) {
    if (res < p->tolerance) return (int)sweep;
    return (int)(sweep + 10 +
                 (unsigned)(p->estimate_sweeps_to_gf_progress * (1.0 - log10(res) / log10(p->tolerance))));
}

static int proxy(gfc_ctx *c, const gfc_params *p, double *res) {
    double e2, th;
    int rc = obs_e2_theta(c, &e2, &th, nullptr);
    if (rc) return rc;
    *res = p->gfix_proxy == GFC_PROXY_THETA ? th : e2;
    return GFC_OK;
}

static void print_res(int sweep, double res) { printf("Sweeps: %8d.\t residue: %3.2E \n", sweep, res); }

// The reference's loop with the exact FP64 kernel and the reference check schedule.
static int fix_reference_schedule(gfc_ctx *c, const gfc_params *p, const gfc_options *o, gfc_report *r) {
    const double omega = (double)p->omega_OR;
    const Lat &l = c->lat;
    int sweep = 0, rc = 0;
    double res;
    int e = proxy(c, p, &res);
    if (e) return e;
    r->initial_residue = res;
    if (o->verbose) print_res(sweep, res);
    int due = next_check(sweep, res, p);
    GFC_CHECK(cudaEventRecord(c->ev_b, c->s));
    while (res > p->tolerance) {
        // half-sweeps up to the next event (scheduled check, max_sweeps, reunitarisation);
        // none of the tests below can fire on the half-sweeps in between
        int n = due - sweep;
        n = std::min(n, (int)p->max_sweeps_to_fix - sweep);
        n = std::min(n, (int)(p->sweeps_to_reunitarization - sweep % p->sweeps_to_reunitarization));
        n = std::max(n, 1);
        if (o->precision == GFC_PREC_FP64_EXACT || l.ns == 1) {
            for (int k = 0; k < n; k++) {
                c->launches += launch_sweep_exact(c->u, c->g, l, sweep + k, omega, p->hits, c->s, c->shape_exact);
            }
        } else {
            // the fast arithmetic; odd ns on the lexicographic layout by boundary levels
            e = l.cb ? halfsweeps_fast64(c, sweep, n, omega, p->hits) : halfsweeps_odd_fast(c, sweep, n, omega, p->hits);
            if (e) return e;
        }
        sweep += n;
        if (sweep == due) {
            double last = res;
            e = proxy(c, p, &res);
            if (e) return e;
            if (fabs(res - last) / last < 10E-16) {
                if (o->verbose) print_res(sweep, res);
                rc = GFC_FIX_NOT_CONVERGED;
                break;
            } else if (res <= p->tolerance) {
                break;
            } else {
                if (o->verbose) print_res(sweep, res);
                due = next_check(sweep, res, p);
            }
        }
        if (sweep >= (int)p->max_sweeps_to_fix) {
            rc = GFC_FIX_NOT_CONVERGED;
            break;
        }
        if (!(sweep % p->sweeps_to_reunitarization)) reunit_spatial_and_g(c);
    }
    GFC_CHECK(cudaEventRecord(c->ev_d, c->s));
    r->site_updates = (long long)sweep * (l.cb ? l.vh : l.v / 2);
    r->sweeps = sweep;
    return rc == 0 ? sweep : rc;
}

// Exact kernel with the proxy evaluated after every half-sweep (standalone
// reduction, one host wait per half-sweep): reference arithmetic, earliest stop.
// Reference arithmetic, the proxy measured exactly (as calculate_e2 / calculateTheta
// do), near the tolerance after every half-sweep.  The test runs on the device: a check kernel after each
// half-sweep's observables sets a stop word, after which the queued sweep and
// observables launches do nothing, so the links returned are those whose proxy was
// found below the tolerance.  The host reads the stop word every 32 half-sweeps and
// reunitarises at the reunitarisation period, which always ends a chunk.
static int fix_every_sweep_exact(gfc_ctx *c, const gfc_params *p, const gfc_options *o, gfc_report *r) {
    const double omega = (double)p->omega_OR;
    const Lat &l = c->lat;
    int sweep = 0;
    double res;
    int e = proxy(c, p, &res);
    if (e) return e;
    r->initial_residue = res;
    if (o->verbose) print_res(sweep, res);
    GFC_CHECK(cudaEventRecord(c->ev_b, c->s));
    if (res <= p->tolerance) {
        GFC_CHECK(cudaEventRecord(c->ev_d, c->s));
        r->sweeps = 0;
        r->first_below_tol = 0;
        return 0;
    }
    unsigned *stop = c->tickets + (l.nt + 1);
    GFC_CHECK(cudaMemsetAsync(stop, 0, sizeof(unsigned), c->s));
    const int theta = p->gfix_proxy == GFC_PROXY_THETA;
    const int max = (int)p->max_sweeps_to_fix, period = (int)p->sweeps_to_reunitarization;
    // The proxy is measured at the end of each chunk while it and its rate put the
    // tolerance more than two chunks away (or it is above 1e3 x tolerance), and after
    // every half-sweep from then on (dense_check: always): the measuring pass costs
    // about as much as a half-sweep.
    unsigned hstop = 0;
    bool dense = o->dense_check != 0;
    int k_a = -1;
    double res_a = 0.0;
    while (sweep < max) {
        int end = std::min(max, sweep + 32);
        if (period > 0) end = std::min(end, (sweep / period + 1) * period);
        for (; sweep < end; sweep++) {
            c->launches += launch_sweep_exact(c->u, c->g, l, sweep, omega, p->hits, c->s, c->shape_exact, stop);
            if (dense || sweep + 1 == end) {
                launch_obs(c->u, l, c->part, c->dres, nullptr, c->s, stop);
                launch_exact_check(c->dres, l, theta, p->tolerance, sweep + 1, stop, c->s);
                c->launches += 3;
            }
        }
        GFC_CHECK(cudaMemcpyAsync(c->hres + 16, stop, sizeof(unsigned), cudaMemcpyDeviceToHost, c->s));
        GFC_CHECK(cudaMemcpyAsync(c->hres + 20, c->dres, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->s));
        GFC_CHECK(cudaStreamSynchronize(c->s));
        GFC_CHECK(cudaGetLastError());
        memcpy(&hstop, c->hres + 16, sizeof hstop);
        if (hstop) break;
        if (!dense) {
            const double res_k = theta ? c->hres[21] / (3.0 * (double)l.v) : c->hres[20] / (double)l.v;
            if (!(res_k == res_k)) break;   // NaN: reported by the final observables
            if (res_k <= 1e3 * p->tolerance) {
                dense = true;
            } else if (k_a >= 0 && res_k < res_a) {
                const double rate = pow(res_k / res_a, 1.0 / (double)(sweep - k_a));
                if (res_k * pow(rate, 64.0) <= 10.0 * p->tolerance) dense = true;
            }
            k_a = sweep;
            res_a = res_k;
        }
        if (period > 0 && !(sweep % period)) reunit_spatial_and_g(c);
    }
    GFC_CHECK(cudaEventRecord(c->ev_d, c->s));
    if (hstop) {
        sweep = (int)hstop;
        r->first_below_tol = sweep;
    }
    r->sweeps = sweep;
    r->site_updates = (long long)sweep * (l.cb ? l.vh : l.v / 2);
    return hstop ? sweep : GFC_FIX_NOT_CONVERGED;
}

extern "C" void gfc_options_default(gfc_options *o) {
    memset(o, 0, sizeof *o);
    o->precision = GFC_PREC_FP64_EXACT;
    o->stop_rule = GFC_STOP_REFERENCE;
    o->verbose = 0;
    o->switch_e2 = 1e-9;
    o->refine_reunit = 0;
    o->block_threads = 0;
}

extern "C" int gfc_ctx_fix(gfc_ctx *c, const gfc_params *p, const gfc_options *opt, gfc_report *rep) {
    if (!c || !p) return GFC_ERR_ARG;
    if (!c->has_links) return GFC_ERR_STATE;
    gfc_options od;
    if (!opt) {
        gfc_options_default(&od);
        opt = &od;
    }
    gfc_report rd;
    gfc_report *r = rep ? rep : &rd;
    memset(r, 0, sizeof *r);
    r->first_below_tol = -1;
    if (!gfc_params_valid(p)) {
        r->status = GFC_FIX_BAD_PARAMS;
        return GFC_FIX_BAD_PARAMS;
    }
    GFC_CHECK(cudaSetDevice(c->dev));
    long long l0 = c->launches;
    const bool mixed = opt->precision == GFC_PREC_MIXED && c->lat.cb;
    if (opt->warm_start && mixed && !c->u0) {
        set_error("context was created without GFC_CTX_MIXED");
        r->status = GFC_ERR_STATE;
        return GFC_ERR_STATE;
    }
    GFC_CHECK(cudaEventRecord(c->ev_a, c->s));
    if (opt->warm_start && mixed) {
        // the mixed path re-gauges the links as uploaded with the whole G at its
        // switch to FP64: keep them before G0 is applied
        GFC_CHECK(cudaMemcpyAsync(c->u0, c->u, (size_t)3 * c->lat.npar * c->lat.vh * 9 * sizeof(double2),
                                  cudaMemcpyDeviceToDevice, c->s));
    }
    if (opt->warm_start) {
        // the resident G is the starting transformation: fix G0 U G0^dagger (spatial
        // links now, temporal ones with the final G at the end) and keep accumulating
        // into G0, so the returned G is the whole transformation of the uploaded links
        launch_apply_gt(c->u, c->ut, c->g, c->lat, 0, c->s);
        c->launches++;
    } else {
        launch_identity(c->g, c->lat, c->s);
        c->launches += c->lat.npar;
    }

    int ret;
    if (mixed) {
        ret = fix_mixed(c, p, opt, r);
    } else if (opt->stop_rule == GFC_STOP_EVERY && (opt->precision == GFC_PREC_FP64_EXACT || c->lat.ns == 1)) {
        ret = fix_every_sweep_exact(c, p, opt, r);
    } else if (opt->stop_rule == GFC_STOP_EVERY && !c->lat.cb) {
        ret = fix_every_sweep_odd_fast(c, p, opt, r);   // odd ns: fast FP64 (no FP32 phase)
    } else if (opt->stop_rule == GFC_STOP_EVERY) {
        ret = fix_every_sweep(c, p, opt, r);
    } else {
        ret = fix_reference_schedule(c, p, opt, r);
    }
    if (ret < GFC_FIX_BAD_PARAMS) return ret;  // a library error, not a fix outcome
    if (ret >= 0) reunit_spatial_and_g(c);
    int e = gfc_ctx_finalize_temporal(c);
    if (e) return e;
    double e2, th, F;
    e = obs_e2_theta(c, &e2, &th, nullptr);
    if (e) return e;
    e = gfc_ctx_functional(c, &F);
    if (e) return e;
    float ms_all = 0, ms_sw = 0;
    GFC_CHECK(cudaEventRecord(c->ev_c, c->s));
    GFC_CHECK(cudaEventSynchronize(c->ev_c));
    // ev_b / ev_d bracket the sweep loop
    GFC_CHECK(cudaEventElapsedTime(&ms_all, c->ev_a, c->ev_c));
    GFC_CHECK(cudaEventElapsedTime(&ms_sw, c->ev_b, c->ev_d));
    r->status = ret;
    r->e2 = e2;
    r->theta = th;
    r->functional = F;
    r->final_residue = p->gfix_proxy == GFC_PROXY_THETA ? th : e2;
    r->seconds_total = ms_all * 1e-3;
    r->seconds_sweeps = ms_sw * 1e-3;
    r->kernel_launches = (int)(c->launches - l0);
    return ret;
}

// gaugefixOverrelaxation(U, G, params) on host arrays in the reference layout
// (src/gauge_fixing.c:713-826, declared include/gauge_fixing.h:67-69): U (4V
// matrices, FP64, native endian) is fixed in place, G (V matrices) receives the
// transformation.  A device context lives for the call.  Returns the reference's
// values: half-sweeps, GFC_FIX_NOT_CONVERGED (-1; U and G are still written, as
// the reference leaves them) or GFC_FIX_BAD_PARAMS (-2; nothing touched); below -2
// a library error.
extern "C" int gfc_gaugefix_overrelaxation(int ns, int nt, double *U, double *G, const gfc_params *p,
                                           const gfc_options *opt, gfc_report *rep, int device) {
    if (!U || !G || !p) return GFC_ERR_ARG;
    if (!gfc_params_valid(p)) return GFC_FIX_BAD_PARAMS;
    gfc_options od;
    if (!opt) {
        gfc_options_default(&od);
        opt = &od;
    }
    gfc_ctx *c = nullptr;
    int rc = gfc_ctx_create(ns, nt, device, opt->precision == GFC_PREC_MIXED ? GFC_CTX_MIXED : 0, &c);
    if (rc) return rc;
    rc = gfc_ctx_upload_links(c, U, 8, 0);
    int fx = rc;
    if (!rc) {
        fx = gfc_ctx_fix(c, p, opt, rep);
        if (fx >= 0 || fx == GFC_FIX_NOT_CONVERGED) {
            rc = gfc_ctx_download_links(c, U, 8, 0);
            if (!rc) rc = gfc_ctx_download_gt(c, G, 8, 0);
            if (rc) fx = rc;
        }
    }
    gfc_ctx_destroy(c);
    return fx;
}
