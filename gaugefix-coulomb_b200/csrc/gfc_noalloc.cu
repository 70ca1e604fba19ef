// gfc_noalloc.cu -- e2 and theta of caller-owned device links with no device
// allocation.
//
// Who needs this: a caller whose device memory is entirely owned by something
// else -- a serving process whose allocator has carved up the whole GPU, or an
// application that sizes every buffer up front -- and a caller that shares the GPU
// with latency-sensitive work on other streams.  Such callers cannot let the
// library call cudaMalloc/cudaFree: an allocation can fail or fragment the
// caller's pool, and cudaFree synchronises the whole device, stalling everyone
// else's streams.  The context API (gfc_ctx_*) allocates its own scratch, so it
// is unusable for them; this entry point takes the links where the caller keeps
// them and uses a fixed scratch array compiled into the library instead.
//
// The scratch is a file-scope __device__ array of GFC_NOALLOC_SCRATCH_DOUBLES
// doubles (128 KiB).  Every GPU that loads the library holds one copy until the
// process exits.  All calls on a GPU share it and it keeps the contents of the
// last call, so two calls whose kernels overlap on the GPU (e.g. issued on two
// streams) race on it and give wrong results: serialise them.  Nothing in it needs
// to start at zero -- each call writes every slot it later reads.
//
// The first call on each device looks up the array's device address
// (cudaGetSymbolAddress) with that device current and caches it.  Every call is
// synchronous: it copies its two sums back to the host and waits for them on
// `stream` before returning.
//
// The links must be device memory of the current device (or managed memory):
// cudaPointerGetAttributes, which allocates nothing, is asked first, and pageable
// or page-locked host memory and another GPU's memory are refused before any
// kernel is launched.
#include <mutex>

#include "gfc.h"
#include "gfc_ctx.h"
#include "gfc_device.cuh"

namespace gfc {

static __device__ __align__(256) double g_noalloc_scratch[GFC_NOALLOC_SCRATCH_DOUBLES];

namespace {

constexpr int NA_BLOCK = 256;
constexpr int NA_MAX_DEVICES = 64;
std::mutex na_mutex;
double *na_scratch[NA_MAX_DEVICES] = {nullptr};

// A_mu = -(i/2) traceless(U - U^dagger), rounded like the reference
// (subtractionHermConjTrless3x3 SU3_ops.c:322-372, calculateA four_potential.c:35-66)
__device__ __forceinline__ void na_calc_A(const M3 &u, M3 &A) {
    M3 d;
    double2 tr = cz();
#pragma unroll
    for (int a = 0; a < 3; a++) {
        d.e[EL(a, a)] = make_double2(0.0, xm(2.0, u.e[EL(a, a)].y));
        tr = xcadd(tr, d.e[EL(a, a)]);
    }
    tr = make_double2(xd(tr.x, 3.0), xd(tr.y, 3.0));
#pragma unroll
    for (int a = 0; a < 3; a++) d.e[EL(a, a)] = xcsub(d.e[EL(a, a)], tr);
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++)
            if (a != b) d.e[EL(a, b)] = xcsub(u.e[EL(a, b)], cconj(u.e[EL(b, a)]));
    const double2 al = make_double2(-0.0, -0.5);
#pragma unroll
    for (int k = 0; k < 9; k++) A.e[k] = xcmul(al, d.e[k]);
}

__device__ __forceinline__ void na_load_aos(const double2 *__restrict__ u, uint32_t L, int mu, M3 &m) {
    const double2 *p = u + ((size_t)L * 4 + mu) * 9;
#pragma unroll
    for (int c = 0; c < 9; c++) m.e[c] = p[c];
}

// e2 density (sum of the 8 algebra components squared, gauge_fixing.c:428-438)
// and theta density (Re Tr divA divA^dagger, gauge_fixing.c:374-380) of site L
__device__ __forceinline__ void na_site(const double2 *__restrict__ u, const Lat &l, uint32_t L, double &e2,
                                        double &th) {
    Coord c = coord_lex(l, L);
    M3 dA;
#pragma unroll
    for (int k = 0; k < 9; k++) dA.e[k] = cz();
#pragma unroll
    for (int d = 0; d < 3; d++) {
        M3 f, r, A1, A2;
        na_load_aos(u, L, d + 1, f);
        na_load_aos(u, back_L(l, c, d), d + 1, r);
        na_calc_A(f, A1);
        na_calc_A(r, A2);
#pragma unroll
        for (int k = 0; k < 9; k++) dA.e[k] = xcadd(dA.e[k], xcsub(A1.e[k], A2.e[k]));
    }
    const double2 *m = dA.e;
    double cc[8];
    cc[0] = xa(m[EL(0, 1)].x, m[EL(1, 0)].x);
    cc[1] = xa(-m[EL(0, 1)].y, m[EL(1, 0)].y);
    cc[2] = xs(m[EL(0, 0)].x, m[EL(1, 1)].x);
    cc[3] = xa(m[EL(0, 2)].x, m[EL(2, 0)].x);
    cc[4] = xa(-m[EL(0, 2)].y, m[EL(2, 0)].y);
    cc[5] = xa(m[EL(1, 2)].x, m[EL(2, 1)].x);
    cc[6] = xa(-m[EL(1, 2)].y, m[EL(2, 1)].y);
    cc[7] = xd(xs(xa(m[EL(0, 0)].x, m[EL(1, 1)].x), xm(2.0, m[EL(2, 2)].x)), __dsqrt_rn(3.0));
    double s = 0.0;
#pragma unroll
    for (int a = 0; a < 8; a++) s = xa(s, xm(cc[a], cc[a]));
    e2 = s;
    double t = 0.0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        double2 sa = cz();
#pragma unroll
        for (int k = 0; k < 3; k++) sa = xcadd(sa, xcmul(m[EL(a, k)], cconj(m[EL(a, k)])));
        t = xa(t, sa.x);
    }
    th = t;
}

// grid (nbx, nt): block bx of timeslice t writes scratch[(t*nbx + bx)*2 + {0,1}]
__global__ void __launch_bounds__(NA_BLOCK) k_obs_partials_noalloc(const double2 *__restrict__ u, Lat l,
                                                                   double *__restrict__ scratch) {
    __shared__ double sh[2][NA_BLOCK / 32];
    const uint32_t t = blockIdx.y;
    double v0 = 0.0, v1 = 0.0;
    for (uint32_t k = blockIdx.x * NA_BLOCK + threadIdx.x; k < l.vs; k += gridDim.x * NA_BLOCK) {
        double e2, th;
        na_site(u, l, t * l.vs + k, e2, th);
        v0 += e2;
        v1 += th;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v0 += __shfl_down_sync(0xffffffffu, v0, o);
        v1 += __shfl_down_sync(0xffffffffu, v1, o);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][wid] = v0;
        sh[1][wid] = v1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0;
        for (int w = 0; w < NA_BLOCK / 32; w++) {
            s0 += sh[0][w];
            s1 += sh[1][w];
        }
        size_t o = ((size_t)t * gridDim.x + blockIdx.x) * 2;
        scratch[o] = s0;
        scratch[o + 1] = s1;
    }
}

// one block: sums the nparts partial pairs in index order into scratch[res_off + {0,1}]
__global__ void __launch_bounds__(NA_BLOCK) k_finalize_noalloc(double *__restrict__ scratch, uint32_t nparts,
                                                               uint32_t res_off) {
    __shared__ double acc[2][NA_BLOCK];
    double s0 = 0.0, s1 = 0.0;
    for (uint32_t p = threadIdx.x; p < nparts; p += NA_BLOCK) {
        s0 += scratch[2 * (size_t)p];
        s1 += scratch[2 * (size_t)p + 1];
    }
    acc[0][threadIdx.x] = s0;
    acc[1][threadIdx.x] = s1;
    __syncthreads();
    for (int w = NA_BLOCK / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            acc[0][threadIdx.x] += acc[0][threadIdx.x + w];
            acc[1][threadIdx.x] += acc[1][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        scratch[res_off] = acc[0][0];
        scratch[res_off + 1] = acc[1][0];
    }
}

// device address of the scratch array on the current device, looked up once
int na_scratch_ptr(double **out) {
    int dev = -1;
    GFC_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NA_MAX_DEVICES) {
        set_error("gfc_e2_theta_device_noalloc: device ordinal %d outside 0..%d", dev, NA_MAX_DEVICES - 1);
        return GFC_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(na_mutex);
    if (!na_scratch[dev]) {
        double *p = nullptr;
        GFC_CHECK(cudaGetSymbolAddress((void **)&p, g_noalloc_scratch));
        na_scratch[dev] = p;
    }
    *out = na_scratch[dev];
    return GFC_OK;
}

}  // namespace
}  // namespace gfc

using namespace gfc;

extern "C" int gfc_e2_theta_device_noalloc(int ns, int nt, const double *u_dev, void *stream, double *e2,
                                           double *theta) {
    if (ns <= 0 || nt <= 0 || !u_dev || !e2 || !theta) {
        set_error("gfc_e2_theta_device_noalloc: bad arguments");
        return GFC_ERR_ARG;
    }
    if ((uintptr_t)u_dev % 16) {
        set_error("gfc_e2_theta_device_noalloc: u_dev must be 16-byte aligned (complex doubles are read in pairs)");
        return GFC_ERR_ARG;
    }
    {
        int cur = -1;
        GFC_CHECK(cudaGetDevice(&cur));
        cudaPointerAttributes pa;
        const cudaError_t pe = cudaPointerGetAttributes(&pa, u_dev);
        if (pe != cudaSuccess) {
            (void)cudaGetLastError();
            set_error("gfc_e2_theta_device_noalloc: u_dev is not a pointer the CUDA runtime knows (%s)",
                      cudaGetErrorString(pe));
            return GFC_ERR_ARG;
        }
        const bool ok = pa.type == cudaMemoryTypeManaged || (pa.type == cudaMemoryTypeDevice && pa.device == cur);
        if (!ok) {
            set_error("gfc_e2_theta_device_noalloc: u_dev must be device memory of the current device %d "
                      "(it is %s memory of device %d)", cur,
                      pa.type == cudaMemoryTypeHost ? "page-locked host"
                      : pa.type == cudaMemoryTypeDevice ? "device" : "unregistered host", pa.device);
            return GFC_ERR_ARG;
        }
    }
    const uint64_t V = (uint64_t)ns * ns * ns * nt;
    if (V * 4 >= (1ull << 31)) {
        set_error("gfc_e2_theta_device_noalloc: lattice %d^3x%d too large for 32-bit site indices", ns, nt);
        return GFC_ERR_GEOMETRY;
    }
    const Lat l = make_lat(ns, nt);
    uint32_t nbx = (l.vs + NA_BLOCK - 1) / NA_BLOCK;
    const uint32_t want = (4u * 148u + (uint32_t)nt - 1) / (uint32_t)nt;
    if (nbx > want) nbx = want;
    if (nbx < 1) nbx = 1;
    const uint64_t nparts = (uint64_t)nbx * (uint64_t)nt;
    const uint64_t res_off = ((2 * nparts + 31) / 32) * 32;   // keep the result 256-byte aligned
    if (res_off + 2 > GFC_NOALLOC_SCRATCH_DOUBLES) {
        set_error("gfc_e2_theta_device_noalloc: nt=%d needs %llu scratch doubles, the fixed scratch holds %d "
                  "(use gfc_ctx_e2 for this lattice)",
                  nt, (unsigned long long)(res_off + 2), GFC_NOALLOC_SCRATCH_DOUBLES);
        return GFC_ERR_ARG;
    }
    double *scratch = nullptr;
    int rc = na_scratch_ptr(&scratch);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    k_obs_partials_noalloc<<<dim3(nbx, nt), NA_BLOCK, 0, s>>>((const double2 *)u_dev, l, scratch);
    k_finalize_noalloc<<<1, NA_BLOCK, 0, s>>>(scratch, (uint32_t)nparts, (uint32_t)res_off);
    GFC_CHECK(cudaGetLastError());
    double h[2];
    GFC_CHECK(cudaMemcpyAsync(h, scratch + res_off, sizeof h, cudaMemcpyDeviceToHost, s));
    GFC_CHECK(cudaStreamSynchronize(s));
    *e2 = h[0] / (double)V;
    *theta = h[1] / (3.0 * (double)V);
    return GFC_OK;
}
