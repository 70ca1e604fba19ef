// gfc_kernels_exact.cu -- FP64 kernels that round exactly like the reference.
//
// k_sweep_exact: one checkerboard half-sweep (gauge_fixing.c:773-787) over the sites
// of one parity, one thread per site.  Each thread builds w(x) from its 3 forward
// and 3 backward spatial links (calculate_w, gauge_fixing.c:445-531), computes the
// over-relaxed update with reference arithmetic (xor_update), and applies it to
// G(x), the 3 forward links and the 3 backward links (updateLocalUG,
// gauge_fixing.c:600-651).  With even ns no two sites of one parity share a link,
// so the parallel half-sweep equals the reference's sequential one bit for bit.
//
// Temporal links are not touched here: they never enter w, e2, theta or F, so
// their transformation is applied once at the end (k_temporal_transform).
//
// Memory traffic per site-update: 6 links + G read and written = 14 x 144 B.
#include "gfc_device.cuh"
#include "gfc.h"
#include "gfc_ctx.h"
#include "gfc_internal.h"

namespace gfc {

template <bool CB>
__device__ __forceinline__ void site_update_exact(double2 *__restrict__ u, double2 *__restrict__ g,
                                                  const Lat &l, int par, const Coord &c, double omega,
                                                  unsigned hits) {
    const int op = CB ? (par ^ 1) : 0;
    const int sp = CB ? par : 0;
    const uint32_t si = CB ? (c.L >> 1) : c.L;
    uint32_t ib[3];
#pragma unroll
    for (int d = 0; d < 3; d++) ib[d] = CB ? (back_L(l, c, d) >> 1) : back_L(l, c, d);

    M3 w;
#pragma unroll
    for (int k = 0; k < 9; k++) w.e[k] = cz();
#pragma unroll
    for (int d = 0; d < 3; d++) {
        M3 f, r;
        load_m(u + uidx(l, d, sp, 0, si), l.vh, f);
        load_m(u + uidx(l, d, op, 0, ib[d]), l.vh, r);
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++)
                w.e[EL(a, b)] = xcadd(w.e[EL(a, b)], xcadd(f.e[EL(a, b)], cconj(r.e[EL(b, a)])));
    }

    M3 upd;
    xor_update(w, omega, hits, upd);

    M3 m, t;
    load_m(g + gidx(l, sp, 0, si), l.vh, m);
    xprod(upd, m, t);
    store_m(g + gidx(l, sp, 0, si), l.vh, t);
#pragma unroll
    for (int d = 0; d < 3; d++) {
        load_m(u + uidx(l, d, sp, 0, si), l.vh, m);
        xprod(upd, m, t);
        store_m(u + uidx(l, d, sp, 0, si), l.vh, t);
        load_m(u + uidx(l, d, op, 0, ib[d]), l.vh, m);
        xprod_dag(m, upd, t);
        store_m(u + uidx(l, d, op, 0, ib[d]), l.vh, t);
    }
}

// Launch shapes (threads per block, minimum resident blocks per SM); the second
// caps registers per thread.  gfc_ctx_autotune picks one per lattice.
// stop (may be null): a stop word set on the device; once it is, the launch does nothing
template <int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) k_sweep_exact(double2 *__restrict__ u, double2 *__restrict__ g,
                                                             Lat l, int par, double omega, unsigned hits,
                                                             const unsigned *stop) {
    if (stop && *(volatile const unsigned *)stop) return;
    uint32_t i = blockIdx.x * BLOCK + threadIdx.x;
    if (i >= l.vh) return;
    Coord c = coord_cb(l, par, i);
    site_update_exact<true>(u, g, l, par, c, omega, hits);
}

// The same update with the six links first copied into shared memory by cp.async
// (9 x 16 B per link per thread: the whole site's links requested at once, no
// registers held for them), read back from there for the link update instead of
// being loaded again.  Arithmetic and order are those of site_update_exact.
// Staged layout: entry e of link m of thread x at sm[(m * 9 + e) * BLOCK + x],
// m = 2d forward, 2d+1 backward link of direction d.  CB = false: the lexicographic
// layout of odd ns (one parity slot, slot index = the site's lexicographic index).
template <int BLOCK, bool CB = true>
__device__ __forceinline__ void site_update_exact_staged(double2 *__restrict__ u, double2 *__restrict__ g,
                                                         const Lat &l, int par, const Coord &c, double omega,
                                                         unsigned hits, double2 *sm) {
    if (!CB) par = 0;
    const int op = CB ? par ^ 1 : 0;
    const uint32_t si = CB ? c.L >> 1 : c.L;
    // G is read only after the update is known: ask for it in L2 now
#pragma unroll
    for (int e = 0; e < 9; e++) asm volatile("prefetch.global.L2 [%0];\n" ::"l"(g + gidx(l, par, e, si)));
    uint32_t ib[3];
#pragma unroll
    for (int d = 0; d < 3; d++) ib[d] = CB ? back_L(l, c, d) >> 1 : back_L(l, c, d);
    double2 *my = sm + threadIdx.x;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double2 *f = u + uidx(l, d, par, 0, si);
        const double2 *r = u + uidx(l, d, op, 0, ib[d]);
#pragma unroll
        for (int e = 0; e < 9; e++) {
            const unsigned sf = (unsigned)__cvta_generic_to_shared(my + ((2 * d) * 9 + e) * BLOCK);
            const unsigned sr = (unsigned)__cvta_generic_to_shared(my + ((2 * d + 1) * 9 + e) * BLOCK);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sf), "l"(f + (size_t)e * l.vh) : "memory");
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sr), "l"(r + (size_t)e * l.vh) : "memory");
        }
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");

    // The direction loops stay rolled: one copy of each body keeps the kernel within
    // the instruction cache (the operands come from shared memory, so no load
    // parallelism is lost); the arithmetic and its order are unchanged.
    M3 w;
#pragma unroll
    for (int k = 0; k < 9; k++) w.e[k] = cz();
#pragma unroll 1
    for (int d = 0; d < 3; d++) {
        M3 f, r;
        load_m(my + (2 * d) * 9 * BLOCK, BLOCK, f);
        load_m(my + (2 * d + 1) * 9 * BLOCK, BLOCK, r);
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++)
                w.e[EL(a, b)] = xcadd(w.e[EL(a, b)], xcadd(f.e[EL(a, b)], cconj(r.e[EL(b, a)])));
    }

    M3 upd;
    xor_update(w, omega, hits, upd);
    asm volatile("" ::: "memory");   // read the links again from shared memory below

    // G is loaded here and multiplied after the six link updates, which hide its
    // latency (the products are independent, so their order changes no result)
    M3 m, t, gm;
    load_m(g + gidx(l, par, 0, si), l.vh, gm);
#pragma unroll 1
    for (int d = 0; d < 3; d++) {
        const uint32_t b = d == 0 ? ib[0] : (d == 1 ? ib[1] : ib[2]);
        load_m(my + (2 * d) * 9 * BLOCK, BLOCK, m);
        xprod(upd, m, t);
        store_m(u + uidx(l, d, par, 0, si), l.vh, t);
        load_m(my + (2 * d + 1) * 9 * BLOCK, BLOCK, m);
        xprod_dag(m, upd, t);
        store_m(u + uidx(l, d, op, 0, b), l.vh, t);
    }
    xprod(upd, gm, t);
    store_m(g + gidx(l, par, 0, si), l.vh, t);
}

template <int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) k_sweep_exact_staged(double2 *__restrict__ u,
                                                                    double2 *__restrict__ g, Lat l, int par,
                                                                    double omega, unsigned hits,
                                                                    const unsigned *stop) {
    extern __shared__ __align__(16) unsigned char exact_stage[];
    if (stop && *(volatile const unsigned *)stop) return;
    uint32_t i = blockIdx.x * BLOCK + threadIdx.x;
    if (i >= l.vh) return;
    Coord c = coord_cb(l, par, i);
    site_update_exact_staged<BLOCK>(u, g, l, par, c, omega, hits, (double2 *)exact_stage);
}

template <int BLOCK, int MINB>
static void launch_exact_staged(const Lat &l, double2 *u, double2 *g, int par, double omega, unsigned hits,
                                cudaStream_t s, const unsigned *stop) {
    constexpr size_t bytes = (size_t)6 * 9 * BLOCK * sizeof(double2);
    static_assert(bytes <= 227 * 1024, "staged links exceed shared memory");
    auto kern = k_sweep_exact_staged<BLOCK, MINB>;
    static std::atomic<unsigned long long> done{0};
    smem_attr_once(done, kern, bytes);
    kern<<<(l.vh + BLOCK - 1) / BLOCK, BLOCK, bytes, s>>>(u, g, l, par, omega, hits, stop);
}

// Odd ns: same-parity sites meet across the periodic boundary, so the updates of a
// half-sweep depend on their order; the reference visits a timeslice in z, y, x
// order (LOOP_SPATIAL).  Two sites of one parity share a link only across the
// boundary: a site with coordinate 0 in direction d and the one with ns - 1 there
// (other coordinates equal), and the reference always updates the first before the
// second.  Ordering the sites by their number of coordinates equal to ns - 1 (the
// boundary level, 0..3) therefore puts every such pair in consecutive levels, in
// the reference's order, and no two sites of one level share a link: sweeping
// level 0, then 1, 2 and 3, each level in parallel, gives every site the links the
// sequential sweep gives it, bit for bit.  Lexicographic layout.
//
// The threads of a launch take the sites of the half-sweep's parity only
// (odd_parity_site): the lanes of a warp are then all of the swept parity (and
// mostly of the launch's level), and the six links of a site are staged in shared
// memory as in the even-ns kernel.
constexpr int LEVEL_BLOCK = 32;
__global__ void __launch_bounds__(LEVEL_BLOCK, 8) k_sweep_exact_level(double2 *__restrict__ u,
                                                                     double2 *__restrict__ g, Lat l, int sweep,
                                                                     int level, double omega, unsigned hits,
                                                                     const unsigned *stop) {
    extern __shared__ __align__(16) unsigned char level_stage[];
    if (stop && *(volatile const unsigned *)stop) return;
    uint32_t L;
    // BLACKRED_SWEEP (gauge_fixing.c:42): parity (x + y + z + t) & 1 = sweep & 1
    if (!odd_parity_site(l, sweep & 1, blockIdx.x * LEVEL_BLOCK + threadIdx.x, L)) return;
    Coord c = coord_lex(l, L);
    const uint32_t e = (uint32_t)l.ns - 1;
    if ((int)(c.x == e) + (int)(c.y == e) + (int)(c.z == e) != level) return;
    // ns = 1: a site's forward and backward link in a direction are one link, updated
    // twice in turn (g U, then that times g^dagger); the unstaged form reads it again
    // between the two, the staged one would not
    if (l.ns == 1)
        site_update_exact<false>(u, g, l, 0, c, omega, hits);
    else
        site_update_exact_staged<LEVEL_BLOCK, false>(u, g, l, 0, c, omega, hits, (double2 *)level_stage);
}

int exact_num_shapes() { return 5; }

// returns the number of kernels launched
int launch_sweep_exact(double2 *u, double2 *g, const Lat &l, int sweep, double omega, unsigned hits,
                        cudaStream_t s, int shape, const unsigned *stop) {
    if (l.cb) {
        int par = sweep & 1;  // BLACKRED_SWEEP: even sites on even sweeps (gauge_fixing.c:42)
        switch (shape) {
            case 1:
                k_sweep_exact<128, 3><<<(l.vh + 127) / 128, 128, 0, s>>>(u, g, l, par, omega, hits, stop);
                break;
            case 2:   // 27 KiB per CTA, 8 CTAs per SM
                launch_exact_staged<32, 8>(l, u, g, par, omega, hits, s, stop);
                break;
            case 3:   // 110.6 KiB of staged links per CTA, 2 CTAs per SM
                launch_exact_staged<128, 2>(l, u, g, par, omega, hits, s, stop);
                break;
            case 4:   // 55.3 KiB per CTA, 4 CTAs per SM
                launch_exact_staged<64, 4>(l, u, g, par, omega, hits, s, stop);
                break;

            default:
                k_sweep_exact<128, 1><<<(l.vh + 127) / 128, 128, 0, s>>>(u, g, l, par, omega, hits, stop);
                break;
        }
    } else {
        // the sites of one parity: ceil(V / 2) at most (V odd when nt is)
        constexpr size_t bytes = (size_t)6 * 9 * LEVEL_BLOCK * sizeof(double2);
        static std::atomic<unsigned long long> done{0};
        smem_attr_once(done, k_sweep_exact_level, bytes);
        const unsigned blocks = (unsigned)((l.v / 2 + 1 + LEVEL_BLOCK - 1) / LEVEL_BLOCK);
        for (int level = 0; level < 4; level++)
            k_sweep_exact_level<<<blocks, LEVEL_BLOCK, bytes, s>>>(u, g, l, sweep, level, omega, hits, stop);
        return 4;
    }
    return 1;
}

// ----------------------------------------------------------- reunitarise --
// reunitarizeField (fields.c:144-187): projectSU3 on every matrix of nmat
// SoA matrices laid out as [c][stride] blocks starting at base + k*9*stride.
__global__ void k_reunitarize(double2 *__restrict__ base, uint32_t stride, uint32_t nblk,
                              unsigned *__restrict__ status) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t k = blockIdx.y;
    if (i >= stride || k >= nblk) return;
    double2 *p = base + (size_t)k * 9 * stride + i;
    M3 m;
    load_m(p, stride, m);
    int st = xproject(m);
    store_m(p, stride, m);
    if (st) atomicOr(status, GFC_STATUS_PROJECT_FAIL);
}

void launch_reunitarize(double2 *base, uint32_t stride, uint32_t nblk, unsigned *status, cudaStream_t s) {
    dim3 grid((stride + 255) / 256, nblk);
    k_reunitarize<<<grid, 256, 0, s>>>(base, stride, nblk, status);
}

__global__ void k_identity(double2 *__restrict__ g, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int c = 0; c < 9; c++) g[(size_t)c * n + i] = make_double2((c % 4) == 0 ? 1.0 : 0.0, 0.0);
}

// G is npar blocks of [9][vh]; treat it as one [9][npar*vh] run per block
void launch_identity(double2 *g, const Lat &l, cudaStream_t s) {
    for (int p = 0; p < l.npar; p++)
        k_identity<<<(l.vh + 255) / 256, 256, 0, s>>>(g + (size_t)p * 9 * l.vh, l.vh);
}

// ------------------------------------------------------------- observables --
// Per site: div A (four_potential.c:70-113) -> e2 density sum_a c_a^2
// (gauge_fixing.c:428-438) and theta density Re Tr(divA divA^dag)
// (gauge_fixing.c:374-380); block partials per timeslice.
__device__ __forceinline__ void calc_A(const M3 &u, M3 &A) {
    // subtractionHermConjTrless3x3 (SU3_ops.c:322-372) then * (-i/2)
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

template <bool CB>
__device__ __forceinline__ void site_obs(const double2 *__restrict__ u, const Lat &l, int par,
                                         const Coord &c, double &e2, double &th) {
    const int op = CB ? (par ^ 1) : 0;
    const int sp = CB ? par : 0;
    const uint32_t si = CB ? (c.L >> 1) : c.L;
    M3 dA;
#pragma unroll
    for (int k = 0; k < 9; k++) dA.e[k] = cz();
#pragma unroll
    for (int d = 0; d < 3; d++) {
        uint32_t Lb = back_L(l, c, d);
        uint32_t ib = CB ? (Lb >> 1) : Lb;
        M3 f, r, A1, A2;
        load_m(u + uidx(l, d, sp, 0, si), l.vh, f);
        load_m(u + uidx(l, d, op, 0, ib), l.vh, r);
        calc_A(f, A1);
        calc_A(r, A2);
#pragma unroll
        for (int k = 0; k < 9; k++) dA.e[k] = xcadd(dA.e[k], xcsub(A1.e[k], A2.e[k]));
    }
    // decomposeAlgebraSU3 (SU3_ops.c:1055-1107)
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
    // Re Tr(dA dA^dag) = sum_ab |dA_ab|^2 accumulated as the trace of prod3x3
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

// block-level deterministic sum of NQ values; result valid in thread 0
template <int NQ>
__device__ __forceinline__ void block_sum(double (&v)[NQ]) {
    __shared__ double sh[NQ][32];
#pragma unroll
    for (int q = 0; q < NQ; q++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NQ; q++) sh[q][wid] = v[q];
    __syncthreads();
    if (wid == 0) {
        int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int q = 0; q < NQ; q++) {
            v[q] = lane < nw ? sh[q][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
        }
    }
    __syncthreads();
}

// grid (nbx, nt): block bx of slice t sums sites of both parities of slice t.  The
// parities alternate from thread to thread (k -> parity k & 1, slot k >> 1): a
// site's backward links are the other parity's, so they are read by a neighbouring
// thread or a recent block and come from L2, not a second time from DRAM, as they
// would if one parity's half of the slice were swept before the other's.
// 128-thread blocks: the six links of a site are all requested at once (~170
// registers), so three blocks (12 warps) fit on an SM where one 256-thread block did
__global__ void __launch_bounds__(128) k_obs_partials(const double2 *__restrict__ u, Lat l,
                                                      double *__restrict__ part, const unsigned *stop) {
    if (stop && *(volatile const unsigned *)stop) return;
    const uint32_t t = blockIdx.y;
    const uint32_t vsh = l.cb ? l.vs / 2 : l.vs;  // slots of one parity per slice
    const uint32_t n = vsh * l.npar;
    double v[2] = {0.0, 0.0};
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int par = l.cb ? (int)(k & 1u) : 0;
        const uint32_t i = t * vsh + (l.cb ? k >> 1 : k);
        double e2, th;
        if (l.cb) {
            Coord c = coord_cb(l, par, i);
            site_obs<true>(u, l, par, c, e2, th);
        } else {
            Coord c = coord_lex(l, i);
            site_obs<false>(u, l, 0, c, e2, th);
        }
        v[0] += e2;
        v[1] += th;
    }
    block_sum<2>(v);
    if (threadIdx.x == 0) {
        size_t o = ((size_t)t * gridDim.x + blockIdx.x) * 2;
        part[o] = v[0];
        part[o + 1] = v[1];
    }
}

// F density: Re Tr of the 3 spatial links at a site (calculateF, gauge_fixing.c:289-337)
__global__ void __launch_bounds__(256) k_functional_partials(const double2 *__restrict__ u, Lat l,
                                                             double *__restrict__ part) {
    const uint32_t t = blockIdx.y;
    const uint32_t vsh = l.cb ? l.vs / 2 : l.vs;
    const uint32_t n = vsh * l.npar;
    double v[1] = {0.0};
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        int par = (int)(k / vsh);
        uint32_t i = t * vsh + (k % vsh);
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const double2 *p = u + uidx(l, d, par, 0, i);
            v[0] += (p[0].x + p[(size_t)4 * l.vh].x) + p[(size_t)8 * l.vh].x;
        }
    }
    block_sum<1>(v);
    if (threadIdx.x == 0) part[(size_t)t * gridDim.x + blockIdx.x] = v[0];
}

// Sum partials [nt][nbx][nq] per slice in a fixed order, then the slices.
// out[q] = total, slice_out[t*nq + q] = per slice (optional).
__global__ void k_finalize(const double *__restrict__ part, int nt, int nbx, int nq, double *__restrict__ out,
                           double *__restrict__ slice_out, const unsigned *stop) {
    if (stop && *(volatile const unsigned *)stop) return;
    __shared__ double acc[4][256];
    for (int q = 0; q < nq; q++) acc[q][threadIdx.x] = 0.0;
    for (int t = threadIdx.x; t < nt; t += blockDim.x) {
        for (int q = 0; q < nq; q++) {
            double s = 0.0;
            for (int b = 0; b < nbx; b++) s += part[((size_t)t * nbx + b) * nq + q];
            if (slice_out) slice_out[(size_t)t * nq + q] = s;
            acc[q][threadIdx.x] += s;
        }
    }
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int q = 0; q < nq; q++) acc[q][threadIdx.x] += acc[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < nq; q++) out[q] = acc[q][0];
}

int obs_blocks_per_slice(const Lat &l) {
    uint32_t vsh = l.cb ? l.vs / 2 : l.vs;
    uint32_t n = vsh * l.npar;
    int nb = (int)((n + 255) / 256);
    // enough blocks overall to fill the GPU, not more than one per 256 sites
    int want = (4 * 148 + l.nt - 1) / l.nt;
    if (nb > want) nb = want;
    if (nb < 1) nb = 1;
    return nb;
}

// sums of nbx per-block (e2, theta) partials per timeslice into out[0..1]
void launch_finalize2(const double *part, const Lat &l, int nbx, double *out, cudaStream_t s, const unsigned *stop) {
    k_finalize<<<1, 256, 0, s>>>(part, l.nt, nbx, 2, out, nullptr, stop);
}

void launch_obs(const double2 *u, const Lat &l, double *part, double *out, double *slice_out, cudaStream_t s,
                const unsigned *stop) {
    int nbx = obs_blocks_per_slice(l);
    k_obs_partials<<<dim3(nbx, l.nt), 128, 0, s>>>(u, l, part, stop);
    k_finalize<<<1, 256, 0, s>>>(part, l.nt, nbx, 2, out, slice_out, stop);
}

// After the observables of half-sweep `sweep`: the proxy (e2 = out[0] / V, or theta =
// out[1] / 3V, normalised as the host does) below the tolerance sets the stop word to
// sweep, once; later sweep and observables launches of the stream then do nothing.
__global__ void k_exact_check(const double *__restrict__ out, double v, int theta, double tol, int sweep,
                              unsigned *stop) {
    if (threadIdx.x || blockIdx.x || *(volatile unsigned *)stop) return;
    const double res = theta ? out[1] / (3.0 * v) : out[0] / v;
    if (res <= tol) *stop = (unsigned)sweep;
}

void launch_exact_check(const double *out, const Lat &l, int theta, double tol, int sweep, unsigned *stop,
                        cudaStream_t s) {
    k_exact_check<<<1, 32, 0, s>>>(out, (double)l.v, theta, tol, sweep, stop);
}

void launch_functional(const double2 *u, const Lat &l, double *part, double *out, cudaStream_t s) {
    int nbx = obs_blocks_per_slice(l);
    k_functional_partials<<<dim3(nbx, l.nt), 256, 0, s>>>(u, l, part);
    k_finalize<<<1, 256, 0, s>>>(part, l.nt, nbx, 1, out, nullptr, nullptr);
}

}  // namespace gfc

// Architecture of the device code the runtime loaded for this library on `device`
// (cudaFuncGetAttributes of one of its kernels): binaryVersion 100 is sm_100 machine
// code, ptxVersion the virtual architecture it was compiled from.
extern "C" int gfc_device_code_version(int device, int *binary_version, int *ptx_version) {
    if (!binary_version || !ptx_version) {
        gfc::set_error("gfc_device_code_version: null output");
        return GFC_ERR_ARG;
    }
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return gfc::cuda_fail(e, "gfc_device_code_version: cudaSetDevice");
    cudaFuncAttributes a;
    e = cudaFuncGetAttributes(&a, gfc::k_identity);
    if (e != cudaSuccess) return gfc::cuda_fail(e, "gfc_device_code_version: cudaFuncGetAttributes");
    *binary_version = a.binaryVersion;
    *ptx_version = a.ptxVersion;
    return GFC_OK;
}

// Self-check of xdiv_shared against IEEE division: count pseudo-random (a, b) pairs,
// significands random or with many trailing zeros or all ones (exact quotients,
// near-ties, the divisors next below powers of two), exponents mostly within a
// factor 2^64 of one and otherwise anywhere (zeros, subnormals, infinities, NaNs).
namespace gfc {
__device__ __forceinline__ uint64_t div_mix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
__device__ double div_operand(uint64_t h, uint64_t form) {
    uint64_t m = h & 0xFFFFFFFFFFFFFULL, e;
    if (form % 5 == 0) m = 0xFFFFFFFFFFFFFULL;
    else if (form % 5 == 1) m = (m >> 30) << 30;
    if ((form >> 3) % 8 == 0) e = (h >> 52) & 0x7FF;          // anywhere
    else e = 1023 - 64 + ((h >> 52) & 127);
    return __longlong_as_double((long long)((h & 0x8000000000000000ULL) | (e << 52) | m));
}
__global__ void k_check_division(uint64_t seed, long long count, unsigned long long *bad) {
    unsigned long long nbad = 0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < count;
         k += (long long)gridDim.x * blockDim.x) {
        const uint64_t h1 = div_mix(seed + 2 * (uint64_t)k), h2 = div_mix(h1 ^ 0x5851F42D4C957F2DULL);
        const uint64_t f = div_mix(h2);
        const double a = div_operand(h1, f), b = div_operand(h2, f >> 8);
        const double want = xd(a, b), got = xdiv_shared(a, b, xrcp(b), xdiv_in_range(b));
        nbad += __double_as_longlong(want) != __double_as_longlong(got);
    }
    if (nbad) atomicAdd(bad, nbad);
}
}  // namespace gfc

extern "C" int gfc_check_division(int device, unsigned long long seed, long long count,
                                  unsigned long long *mismatches) {
    if (!mismatches || count < 0) {
        gfc::set_error("gfc_check_division: null output or negative count");
        return GFC_ERR_ARG;
    }
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return gfc::cuda_fail(e, "gfc_check_division: cudaSetDevice");
    unsigned long long *d = nullptr;
    if ((e = cudaMalloc(&d, sizeof *d)) != cudaSuccess) return gfc::cuda_fail(e, "gfc_check_division: cudaMalloc");
    if ((e = cudaMemset(d, 0, sizeof *d)) == cudaSuccess) {
        gfc::k_check_division<<<148 * 8, 256>>>(seed, count, d);
        if ((e = cudaGetLastError()) == cudaSuccess && (e = cudaDeviceSynchronize()) == cudaSuccess)
            e = cudaMemcpy(mismatches, d, sizeof *d, cudaMemcpyDeviceToHost);
    }
    cudaFree(d);
    return e == cudaSuccess ? GFC_OK : gfc::cuda_fail(e, "gfc_check_division");
}
