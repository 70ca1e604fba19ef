// gfc_kernels_io.cu -- layout/precision/endianness transforms and observables that
// run once per fix (not per half-sweep).
//
//  * k_load_links: the reference's loadConfig (fields_io.c:216-305) after the raw
//    bytes are on the device: byte swap of 8- or 4-byte words (byteSwap,
//    fields_io.c:42-96), FP32 -> FP64 (convertCfg_in_work,
//    convert_precision_io.c:176-215), AoS -> checkerboard SoA, temporal links split
//    off.  One pass over timeslice chunks, so the host can stream the file in.
//  * k_store_gt / k_store_links: writeGaugeTransf / writeConfig
//    (fields_io.c:405-565) in the other direction, optional FP32 output
//    (convertGT_work_out / convertCfg_work_out) and optional byte swap.
//  * k_temporal_transform: U_t(x) <- G(x) U_t(x) G(x+t)^dagger once at the end;
//    the reference applies the same product incrementally every half-sweep
//    (updateLocalUG, gauge_fixing.c:638-650) although temporal links never feed
//    back into the update.
//  * k_plaquette_partials: averagePlaquette (measurement.c:37-155).
#include "gfc_device.cuh"
#include "gfc_internal.h"

namespace gfc {

__device__ __forceinline__ double load_elem(const void *raw, size_t e, int elem_bytes, int swap) {
    if (elem_bytes == 8) {
        uint2 w = reinterpret_cast<const uint2 *>(raw)[e];
        if (swap) {
            uint32_t lo = __byte_perm(w.y, 0, 0x0123), hi = __byte_perm(w.x, 0, 0x0123);
            w.x = lo;
            w.y = hi;
        }
        return __hiloint2double((int)w.y, (int)w.x);
    }
    uint32_t w = reinterpret_cast<const uint32_t *>(raw)[e];
    if (swap) w = __byte_perm(w, 0, 0x0123);
    return (double)__uint_as_float(w);
}

__device__ __forceinline__ void store_elem(void *raw, size_t e, int elem_bytes, int swap, double v) {
    if (elem_bytes == 8) {
        uint32_t lo = (uint32_t)__double2loint(v), hi = (uint32_t)__double2hiint(v);
        if (swap) {
            uint32_t nlo = __byte_perm(hi, 0, 0x0123), nhi = __byte_perm(lo, 0, 0x0123);
            lo = nlo;
            hi = nhi;
        }
        reinterpret_cast<uint2 *>(raw)[e] = make_uint2(lo, hi);
        return;
    }
    uint32_t w = __float_as_uint((float)v);
    if (swap) w = __byte_perm(w, 0, 0x0123);
    reinterpret_cast<uint32_t *>(raw)[e] = w;
}

// one thread per (site, mu) of the chunk; raw holds the chunk only
// With reunit != 0 each matrix is also projected to SU(3) (projectSU3, the reference
// arithmetic of k_reunitarize) before it is stored: loadConfig and reunitarizeField
// (gauge_fix_coulomb.c:123-131) in one pass over the links.
__global__ void k_load_links(const void *__restrict__ raw, int elem_bytes, int swap, Lat l, uint32_t t0,
                             uint32_t nts, double2 *__restrict__ u, double2 *__restrict__ ut, int reunit,
                             unsigned *__restrict__ status) {
    size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    size_t nmat = (size_t)nts * l.vs * 4;
    if (k >= nmat) return;
    uint32_t L = t0 * l.vs + (uint32_t)(k >> 2);
    int mu = (int)(k & 3);
    Slot s = slot_of(l, L);
    double2 *dst = mu == 0 ? ut + gidx(l, s.par, 0, s.i) : u + uidx(l, mu - 1, s.par, 0, s.i);
    M3 m;
#pragma unroll
    for (int c = 0; c < 9; c++) {
        double re = load_elem(raw, k * 18 + 2 * c, elem_bytes, swap);
        double im = load_elem(raw, k * 18 + 2 * c + 1, elem_bytes, swap);
        m.e[c] = make_double2(re, im);
    }
    if (reunit && xproject(m)) atomicOr(status, GFC_STATUS_PROJECT_FAIL);
    store_m(dst, l.vh, m);
}

void launch_load_links(const void *raw, int elem_bytes, int swap, const Lat &l, uint32_t t0, uint32_t nts,
                       double2 *u, double2 *ut, cudaStream_t s, int reunit, unsigned *status) {
    size_t n = (size_t)nts * l.vs * 4;
    k_load_links<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(raw, elem_bytes, swap, l, t0, nts, u, ut, reunit,
                                                               status);
}

__global__ void k_store_gt(const double2 *__restrict__ g, Lat l, uint32_t t0, uint32_t nts, int elem_bytes,
                           int swap, void *__restrict__ raw) {
    size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (size_t)nts * l.vs) return;
    Slot s = slot_of(l, t0 * l.vs + (uint32_t)k);
    const double2 *src = g + gidx(l, s.par, 0, s.i);
#pragma unroll
    for (int c = 0; c < 9; c++) {
        double2 v = src[(size_t)c * l.vh];
        store_elem(raw, k * 18 + 2 * c, elem_bytes, swap, v.x);
        store_elem(raw, k * 18 + 2 * c + 1, elem_bytes, swap, v.y);
    }
}

void launch_store_gt(const double2 *g, const Lat &l, uint32_t t0, uint32_t nts, int elem_bytes, int swap,
                     void *raw, cudaStream_t s) {
    size_t n = (size_t)nts * l.vs;
    k_store_gt<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(g, l, t0, nts, elem_bytes, swap, raw);
}

__global__ void k_load_gt(const void *__restrict__ raw, int elem_bytes, int swap, Lat l, uint32_t t0,
                          uint32_t nts, double2 *__restrict__ g) {
    size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (size_t)nts * l.vs) return;
    Slot s = slot_of(l, t0 * l.vs + (uint32_t)k);
    double2 *dst = g + gidx(l, s.par, 0, s.i);
#pragma unroll
    for (int c = 0; c < 9; c++) {
        double re = load_elem(raw, k * 18 + 2 * c, elem_bytes, swap);
        double im = load_elem(raw, k * 18 + 2 * c + 1, elem_bytes, swap);
        dst[(size_t)c * l.vh] = make_double2(re, im);
    }
}

void launch_load_gt(const void *raw, int elem_bytes, int swap, const Lat &l, uint32_t t0, uint32_t nts,
                    double2 *g, cudaStream_t s) {
    size_t n = (size_t)nts * l.vs;
    k_load_gt<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(raw, elem_bytes, swap, l, t0, nts, g);
}

__global__ void k_store_links(const double2 *__restrict__ u, const double2 *__restrict__ ut, Lat l,
                              uint32_t t0, uint32_t nts, int elem_bytes, int swap, void *__restrict__ raw) {
    size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (size_t)nts * l.vs * 4) return;
    uint32_t L = t0 * l.vs + (uint32_t)(k >> 2);
    int mu = (int)(k & 3);
    Slot s = slot_of(l, L);
    const double2 *src = mu == 0 ? ut + gidx(l, s.par, 0, s.i) : u + uidx(l, mu - 1, s.par, 0, s.i);
#pragma unroll
    for (int c = 0; c < 9; c++) {
        double2 v = src[(size_t)c * l.vh];
        store_elem(raw, k * 18 + 2 * c, elem_bytes, swap, v.x);
        store_elem(raw, k * 18 + 2 * c + 1, elem_bytes, swap, v.y);
    }
}

void launch_store_links(const double2 *u, const double2 *ut, const Lat &l, uint32_t t0, uint32_t nts,
                        int elem_bytes, int swap, void *raw, cudaStream_t s) {
    size_t n = (size_t)nts * l.vs * 4;
    k_store_links<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(u, ut, l, t0, nts, elem_bytes, swap, raw);
}

// U'(x) = G(x) U(x) G(y)^dagger with the products rounded like prod_vuwdagger3x3
// (SU3_ops.c:703-730) would round a two-step product
__device__ __forceinline__ void gug(const M3 &gx, const M3 &uu, const M3 &gy, M3 &out) {
    M3 t;
    xprod(gx, uu, t);
    xprod_dag(t, gy, out);
}

__global__ void k_temporal_transform(double2 *__restrict__ ut, const double2 *__restrict__ g, Lat l) {
    uint32_t L = blockIdx.x * blockDim.x + threadIdx.x;
    if (L >= l.v) return;
    Coord c = coord_lex(l, L);
    Slot s = slot_of(l, L), sy = slot_of(l, fwd_t_L(l, c));
    M3 gx, gy, uu, o;
    load_m(g + gidx(l, s.par, 0, s.i), l.vh, gx);
    load_m(g + gidx(l, sy.par, 0, sy.i), l.vh, gy);
    load_m(ut + gidx(l, s.par, 0, s.i), l.vh, uu);
    gug(gx, uu, gy, o);
    store_m(ut + gidx(l, s.par, 0, s.i), l.vh, o);
}

void launch_temporal_transform(double2 *ut, const double2 *g, const Lat &l, cudaStream_t s) {
    k_temporal_transform<<<(l.v + 127) / 128, 128, 0, s>>>(ut, g, l);
}

__global__ void k_apply_gt_spatial(double2 *__restrict__ u, const double2 *__restrict__ u0,
                                   const double2 *__restrict__ g, Lat l) {
    uint32_t L = blockIdx.x * blockDim.x + threadIdx.x;
    if (L >= l.v) return;
    Coord c = coord_lex(l, L);
    Slot s = slot_of(l, L);
    M3 gx;
    load_m(g + gidx(l, s.par, 0, s.i), l.vh, gx);
#pragma unroll
    for (int d = 0; d < 3; d++) {
        Slot sy = slot_of(l, fwd_L(l, c, d));
        M3 gy, uu, o;
        load_m(g + gidx(l, sy.par, 0, sy.i), l.vh, gy);
        load_m(u0 + uidx(l, d, s.par, 0, s.i), l.vh, uu);
        gug(gx, uu, gy, o);
        store_m(u + uidx(l, d, s.par, 0, s.i), l.vh, o);
    }
}

// prod_vuwdagger3x3 (SU3_ops.c:688-730) in its own order: o_ab = sum_c sum_d
// (v_ac u_cd) conj(w_bd), accumulated from zero, every product and sum rounded alone
__device__ __forceinline__ void xvuwdag(const M3 &v, const M3 &u, const M3 &w, M3 &o) {
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
            double2 s = cz();
#pragma unroll
            for (int c = 0; c < 3; c++)
#pragma unroll
                for (int d = 0; d < 3; d++)
                    s = xcadd(s, xcmul(xcmul(v.e[EL(a, c)], u.e[EL(c, d)]), cconj(w.e[EL(b, d)])));
            o.e[EL(a, b)] = s;
        }
}

// applyGaugeTransformationU (fields.c:375-435), in place: U_mu(x) <- G(x) U_mu(x)
// G(x+mu)^dagger for the spatial links and, with temporal != 0, the temporal ones.
// Each thread reads and writes only the links of its own site.
__global__ void k_apply_gt(double2 *__restrict__ u, double2 *__restrict__ ut, const double2 *__restrict__ g,
                           Lat l, int temporal) {
    uint32_t L = blockIdx.x * blockDim.x + threadIdx.x;
    if (L >= l.v) return;
    Coord c = coord_lex(l, L);
    Slot s = slot_of(l, L);
    M3 gx, gy, uu, o;
    load_m(g + gidx(l, s.par, 0, s.i), l.vh, gx);
    if (temporal) {
        Slot sy = slot_of(l, fwd_t_L(l, c));
        load_m(g + gidx(l, sy.par, 0, sy.i), l.vh, gy);
        load_m(ut + gidx(l, s.par, 0, s.i), l.vh, uu);
        xvuwdag(gx, uu, gy, o);
        store_m(ut + gidx(l, s.par, 0, s.i), l.vh, o);
    }
#pragma unroll 1
    for (int d = 0; d < 3; d++) {
        Slot sy = slot_of(l, fwd_L(l, c, d));
        load_m(g + gidx(l, sy.par, 0, sy.i), l.vh, gy);
        load_m(u + uidx(l, d, s.par, 0, s.i), l.vh, uu);
        xvuwdag(gx, uu, gy, o);
        store_m(u + uidx(l, d, s.par, 0, s.i), l.vh, o);
    }
}

void launch_apply_gt(double2 *u, double2 *ut, const double2 *g, const Lat &l, int temporal, cudaStream_t s) {
    k_apply_gt<<<(l.v + 127) / 128, 128, 0, s>>>(u, ut, g, l, temporal);
}

void launch_apply_gt_spatial(double2 *u, const double2 *u0, const double2 *g, const Lat &l, cudaStream_t s) {
    k_apply_gt_spatial<<<(l.v + 127) / 128, 128, 0, s>>>(u, u0, g, l);
}

// ---------------------------------------------------------------- plaquette --
__device__ __forceinline__ const double2 *link_ptr(const double2 *u, const double2 *ut, const Lat &l, int mu,
                                                   uint32_t L) {
    Slot s = slot_of(l, L);
    return mu == 0 ? ut + gidx(l, s.par, 0, s.i) : u + uidx(l, mu - 1, s.par, 0, s.i);
}
__device__ __forceinline__ uint32_t fwd_mu(const Lat &l, uint32_t L, int mu) {
    Coord c = coord_lex(l, L);
    return mu == 0 ? fwd_t_L(l, c) : fwd_L(l, c, mu - 1);
}

// Re Tr(U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag) / 3  (TrPlaquette, measurement.c:37-75)
__device__ double plaq(const double2 *u, const double2 *ut, const Lat &l, uint32_t L, int mu, int nu) {
    uint32_t Lm = fwd_mu(l, L, mu), Ln = fwd_mu(l, L, nu);
    M3 a, b, c, d, ab, cd;
    load_m(link_ptr(u, ut, l, mu, L), l.vh, a);
    load_m(link_ptr(u, ut, l, nu, Lm), l.vh, b);
    load_m(link_ptr(u, ut, l, mu, Ln), l.vh, c);
    load_m(link_ptr(u, ut, l, nu, L), l.vh, d);
    xprod(a, b, ab);
    // cd = c^dag d^dag = (d c)^dag
    M3 dc;
    xprod(d, c, dc);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) cd.e[EL(i, j)] = cconj(dc.e[EL(j, i)]);
    double tr = 0.0;
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) tr = xa(tr, xcmul(ab.e[EL(i, k)], cd.e[EL(k, i)]).x);
    return xd(tr, 3.0);
}

__device__ __forceinline__ void block_sum2(double &a, double &b) {
    __shared__ double sh[2][32];
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][wid] = a;
        sh[1][wid] = b;
    }
    __syncthreads();
    if (wid == 0) {
        int nw = (blockDim.x + 31) >> 5;
        a = lane < nw ? sh[0][lane] : 0.0;
        b = lane < nw ? sh[1][lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
    }
    __syncthreads();
}

__global__ void __launch_bounds__(256) k_plaquette_partials(const double2 *__restrict__ u,
                                                            const double2 *__restrict__ ut, Lat l,
                                                            double *__restrict__ part) {
    const uint32_t t = blockIdx.y;
    double sp = 0.0, tp = 0.0;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < l.vs; k += gridDim.x * blockDim.x) {
        uint32_t L = t * l.vs + k;
        for (int i = 1; i <= 3; i++) tp += plaq(u, ut, l, L, 0, i);
        sp += plaq(u, ut, l, L, 3, 2);
        sp += plaq(u, ut, l, L, 3, 1);
        sp += plaq(u, ut, l, L, 2, 1);
    }
    block_sum2(sp, tp);
    if (threadIdx.x == 0) {
        size_t o = ((size_t)t * gridDim.x + blockIdx.x) * 2;
        part[o] = sp;
        part[o + 1] = tp;
    }
}

__global__ void k_finalize2(const double *__restrict__ part, int nt, int nbx, double *__restrict__ out) {
    __shared__ double acc[2][256];
    acc[0][threadIdx.x] = 0.0;
    acc[1][threadIdx.x] = 0.0;
    for (int t = threadIdx.x; t < nt; t += blockDim.x)
        for (int q = 0; q < 2; q++) {
            double s = 0.0;
            for (int b = 0; b < nbx; b++) s += part[((size_t)t * nbx + b) * 2 + q];
            acc[q][threadIdx.x] += s;
        }
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            acc[0][threadIdx.x] += acc[0][threadIdx.x + w];
            acc[1][threadIdx.x] += acc[1][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = acc[0][0];
        out[1] = acc[1][0];
    }
}

void launch_plaquette(const double2 *u, const double2 *ut, const Lat &l, double *part, double *out,
                      cudaStream_t s) {
    int nbx = obs_blocks_per_slice(l);
    k_plaquette_partials<<<dim3(nbx, l.nt), 256, 0, s>>>(u, ut, l, part);
    k_finalize2<<<1, 256, 0, s>>>(part, l.nt, nbx, out);
}

}  // namespace gfc
