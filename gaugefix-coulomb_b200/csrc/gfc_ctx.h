// gfc_ctx.h -- the device-resident state behind a gfc_ctx handle.
#pragma once
#include <cuda_runtime.h>
#include <stdio.h>

#include "gfc.h"
#include "gfc_internal.h"

struct gfc_ctx {
    int dev = 0;
    gfc::Lat lat{};
    cudaStream_t s = nullptr;     // compute stream (all kernels)
    cudaStream_t sc = nullptr;    // copy stream (chunked host <-> device)
    // FP64 fields (checkerboard SoA, see gfc_device.cuh)
    double2 *u = nullptr;         // spatial links, 3 directions
    double2 *g = nullptr;         // gauge transformation
    double2 *ut = nullptr;        // temporal links
    double2 *u0 = nullptr;        // copy of the spatial links at the start of a mixed fix
    void *backup = nullptr;       // gfc_ctx_save_links copy (spatial + temporal)
    double2 *u64r = nullptr;      // fast FP64 sweeps: links, rows 0 and 1 only
    double2 *g64r = nullptr;      // fast FP64 sweeps: G, rows 0 and 1 only
    // FP32 fields for the mixed-precision bulk (two stored rows per link)
    float2 *u32 = nullptr;
    float2 *g32 = nullptr;
    // reduction scratch and device scalars
    double *part = nullptr;
    size_t part_n = 0;
    double *dres = nullptr;       // [32] device results
    double *hres = nullptr;       // [32] pinned mirror
    unsigned *dstatus = nullptr;
    double *e2_slice = nullptr;   // [nt] per-timeslice e2 partials (fused path)
    double *e2_hist = nullptr;    // [2][hist_n] per half-sweep fused e2 (two parity halves)
    int hist_n = 0;
    // chunked I/O staging
    size_t stage_bytes = 0;
    void *dstage[2] = {nullptr, nullptr};
    void *hstage[2] = {nullptr, nullptr};
    cudaEvent_t ev_copy[2] = {nullptr, nullptr}, ev_used[2] = {nullptr, nullptr};
    cudaEvent_t ev_a = nullptr, ev_b = nullptr, ev_c = nullptr, ev_d = nullptr;
    unsigned *tickets = nullptr;  // [nt + 2]: per-slice and global tickets, stop word
    int has_links = 0;
    long long launches = 0;
    // launch shapes of the sweep kernels (indices into the compiled shape tables;
    // defaults until gfc_ctx_autotune measures them for this lattice)
    // (the defaults are the shapes the autotuner picks at 32^3x64 on a B200: exact with
    // the links staged in blocks of 64 sites, 4 per SM (368-376 us per half-sweep);
    // fast FP64 and FP32 with links and G staged in blocks of 64 sites, 5 per SM
    // (215-216 us and 111-112 us; the plain FP32 128 x 5 shape takes 127-129 us))
    int shape_exact = 4;
    int shape_fast64 = 10;
    int shape_fast32 = 10;
    int tuned = 0;
    // slice blocking of the fast sweeps: groups of blk*_slices timeslices run
    // blk*_sweeps half-sweeps each while resident in L2 (0 / 1: not blocked)
    int blk64_slices = 0, blk64_sweeps = 1;
    int blk32_slices = 0, blk32_sweeps = 1;
    double *ring = nullptr;       // per-slice e2 partials of the last half-sweeps
    int ring_n = 0;
};

namespace gfc {
void set_error(const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);
}  // namespace gfc

#define GFC_CHECK(call)                                                   \
    do {                                                                  \
        cudaError_t _e = (call);                                          \
        if (_e != cudaSuccess) return gfc::cuda_fail(_e, #call);          \
    } while (0)
