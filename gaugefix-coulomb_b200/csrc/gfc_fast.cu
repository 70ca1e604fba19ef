// gfc_fast.cu -- bandwidth-oriented sweep kernels, fused gauge-functional
// reductions, and the every-half-sweep and mixed-precision drivers.
//
// The update is the reference's over-relaxation (gauge_fixing.c:656-708) computed
// the direct way: the Cabibbo-Marinari SU(2) rotations are applied to w and, at the
// same time, accumulated into the update g, so g = w_final . w^-1 without forming
// the explicit 3x3 inverse and its 18 divisions.  FMA contraction is allowed.
//
// Fused e2.  With D = w - w^dagger, div A(x) = (-i/2) traceless(D) (expand
// four_potential.c:70-113 in terms of w from gauge_fixing.c:491-531), so the e2
// density of a site is a function of w(x) alone:
//   c1 = Im w01 + Im w10, c2 = Re w01 - Re w10, c3 = Im w00 - Im w11,
//   c4 = Im w02 + Im w20, c5 = Re w02 - Re w20, c6 = Im w12 + Im w21,
//   c7 = Re w12 - Re w21, c8 = (Im w00 + Im w11 - 2 Im w22)/sqrt(3).
// A half-sweep of parity p reads w of every parity-p site before its update (the
// state after the previous half-sweep) and, from the six links it has just
// written, w after its update.  e2 after half-sweep k is therefore
//   post(k) [parity-p sites, kernel k] + pre(k+1) [other sites, kernel k+1],
// available inside kernel k+1 with no extra pass over memory.  Per-block partials
// are combined per timeslice and then over timeslices by the last block to
// finish (fixed summation order, so the result does not depend on scheduling).
// When the stopping test fires, that block writes the stop word and every later
// kernel of the same stream returns at entry.
//
// Storage policies:
//   S64: FP64, all 9 entries (double2 per entry), 144 B per matrix.
//   S32: FP32, rows 0 and 1 only (3 float4), 48 B per matrix; row 2 is rebuilt as
//        conj(row0 x row1), which is exact for SU(3).
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>

#include "gfc_device.cuh"
#include "gfc_fast.h"

#include "gfc_fast_device.cuh"

namespace gfc {

// ----------------------------------------------------------- sweep kernel --
struct SweepArgs {
    Lat l;
    int par;
    double omega;
    unsigned hits;
    int track;          // 0: none; 1: per-slice + whole-lattice sums and stop test
                        // (grid covers all slices); 2: per-slice sums into the ring only
    int t0;             // first timeslice of this launch (grid.y slices from t0)
    double *part;       // [nt][nbx][2]
    unsigned *tickets;  // [nt + 1]
    double *slice;      // [nt][2] latest per-slice (pre, post) sums
    double *ring;       // track 2: [ring_n][nt][2] per-slice sums by half-sweep index
    int ring_n;
    double *hist;       // [2 * hist_n]: (pre, post) totals per sweep index
    int sweep;          // this half-sweep's index
    int hist_n;
    unsigned *stop;     // stop word (0 = keep going); nullptr = never stop
    double tol_sum;     // stop when post(sweep-1) + pre(sweep) <= tol_sum
    int test;           // 1: hist holds post(sweep-1) of this run, so the stop test applies
    unsigned *status;
    int proj;           // 1: project the links written onto SU(3) (reunitarisation folded in;
                        // honoured by the fully staged two-row shapes, see links_fold_reunit)
};

// Launch shapes compiled into the library: (threads per block, minimum resident
// blocks per SM).  The second number caps registers per thread (65536 / (block *
// minb)); which shape is fastest depends on the lattice and is measured by
// gfc_ctx_autotune.
struct Shape {
    int block, minb;
};
constexpr Shape kShapes[] = {{128, 2}, {128, 3}, {128, 4}, {64, 4}, {64, 6}, {256, 1}, {256, 2}, {128, 5}, {128, 6}};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);
// Shapes of the shared-memory staged kernel (two-row storage only): the six links
// and, with sg, G are copied to shared memory by cp.async before the update
// (6 or 7 x 96 B per thread in FP64, 48 B in FP32), which also bounds residency.
struct SShape {
    int block, minb, sg, nst;   // nst: links staged per site (whole directions: 2, 4 or 6)
};
constexpr SShape kStaged[] = {{128, 2, 1, 6}, {64, 5, 1, 6}, {128, 3, 0, 6}, {64, 6, 0, 6}, {32, 11, 0, 6},
                              {32, 12, 0, 6}, {64, 7, 0, 4}, {128, 4, 0, 4}, {128, 4, 0, 2}};
constexpr int kNumStaged = sizeof(kStaged) / sizeof(kStaged[0]);
constexpr int kNumAll = kNumShapes + kNumStaged;   // shape indices: plain, then staged
constexpr int kNE = 5;   // exact-kernel shapes (gfc_kernels_exact.cu)
static_assert(kNE + 2 * kNumAll + 8 == GFC_TUNE_SLOTS, "autotune time slots");
constexpr int MIN_BLOCK = 32;   // smallest block: sizes the per-block partial buffers

// deterministic sum of NQ values over the block; result in thread 0
template <int BLOCK, int NQ>
__device__ __forceinline__ void fblock_sum(double (&v)[NQ], double (*sh)[BLOCK / 32]) {
#pragma unroll
    for (int q = 0; q < NQ; q++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NQ; q++) sh[q][wid] = v[q];
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < NQ; q++) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < BLOCK / 32; k++) s += sh[q][k];
            v[q] = s;
        }
}

// Combine block partials: last block of a slice sums the slice, last slice sums
// all slices, applies the stopping test.  Called by all threads of the block; sh and
// last are shared-memory scratch of the block.
template <int BLOCK>
__device__ void fused_reduce(const SweepArgs &a, double pre, double post, double (*sh)[BLOCK / 32], int &last) {
    double v[2] = {pre, post};
    fblock_sum<BLOCK, 2>(v, sh);
    const uint32_t t = a.t0 + blockIdx.y, nbx = gridDim.x, nt = gridDim.y;
    if (threadIdx.x == 0) {
        size_t o = ((size_t)t * nbx + blockIdx.x) * 2;
        a.part[o] = v[0];
        a.part[o + 1] = v[1];
        __threadfence();
        unsigned tk = atomicAdd(&a.tickets[t], 1u);
        last = tk == nbx - 1;
    }
    __syncthreads();
    if (!last) return;
    // slice sum: each thread a fixed strided share of the partials, then the block
    // tree (a fixed order, so the result does not depend on which block came last)
    {
        const double *p = a.part + (size_t)t * nbx * 2;
        v[0] = v[1] = 0.0;
        for (uint32_t b = threadIdx.x; b < nbx; b += BLOCK) {
            v[0] += __ldcg(p + 2 * b);
            v[1] += __ldcg(p + 2 * b + 1);
        }
        fblock_sum<BLOCK, 2>(v, sh);
    }
    if (threadIdx.x == 0) {
        a.tickets[t] = 0;
        if (a.track == 2) {
            // slice-blocked sweeping: the whole-lattice test runs after the round
            double *r = a.ring + ((size_t)(a.sweep % a.ring_n) * a.l.nt + t) * 2;
            r[0] = v[0];
            r[1] = v[1];
            last = 0;
        } else {
            a.slice[2 * t] = v[0];
            a.slice[2 * t + 1] = v[1];
            __threadfence();
            unsigned tk = atomicAdd(&a.tickets[nt], 1u);
            last = tk == nt - 1;
        }
    }
    __syncthreads();
    if (!last) return;
    v[0] = v[1] = 0.0;
    for (uint32_t q = threadIdx.x; q < nt; q += BLOCK) {
        v[0] += __ldcg(a.slice + 2 * q);
        v[1] += __ldcg(a.slice + 2 * q + 1);
    }
    fblock_sum<BLOCK, 2>(v, sh);
    if (threadIdx.x != 0) return;
    const double s0 = v[0], s1 = v[1];
    a.tickets[nt] = 0;
    if (a.sweep < a.hist_n) {
        a.hist[2 * a.sweep] = s0;
        a.hist[2 * a.sweep + 1] = s1;
    }
    if (!(s0 == s0) || !(s1 == s1)) {
        atomicOr(a.status, GFC_STATUS_NAN);
        if (a.stop) atomicExch(a.stop, 0x80000000u | (unsigned)(a.sweep + 1));
        return;
    }
    if (a.stop && a.test && a.sweep >= 1 && a.sweep - 1 < a.hist_n) {
        double e2 = __ldcg(a.hist + 2 * (a.sweep - 1) + 1) + s0;
        if (e2 <= a.tol_sum) atomicExch(a.stop, (unsigned)(a.sweep + 1));
    }
}

template <class S, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) k_sweep_fast(typename S::V *__restrict__ u,
                                                            typename S::V *__restrict__ g, SweepArgs a) {
    using T = typename S::T;
    if (a.stop && *(volatile unsigned *)a.stop) return;
    const Lat &l = a.l;
    const uint32_t vsh = l.vs >> 1;
    const uint32_t off = blockIdx.x * BLOCK + threadIdx.x;
    const bool active = off < vsh;
    double pre = 0.0, post = 0.0;
    if (active) fast_site<S>(u, g, l, a.par, (a.t0 + blockIdx.y) * vsh + off, (T)a.omega, a.hits, a.track, pre, post);
    __shared__ double sh[2][BLOCK / 32];
    __shared__ int last;
    if (a.track) fused_reduce<BLOCK>(a, pre, post, sh, last);
}

template <class S, int BLOCK, int MINB, bool SG, int NST, bool PROJ = false>
__global__ void __launch_bounds__(BLOCK, MINB) k_sweep_staged(typename S::V *__restrict__ u,
                                                              typename S::V *__restrict__ g, SweepArgs a) {
    extern __shared__ __align__(16) unsigned char staged_smem[];
    using T = typename S::T;
    if (a.stop && *(volatile unsigned *)a.stop) return;
    const Lat &l = a.l;
    const uint32_t vsh = l.vs >> 1;
    const uint32_t off = blockIdx.x * BLOCK + threadIdx.x;
    double pre = 0.0, post = 0.0;
    if (off < vsh)
        fast_site_staged<S, BLOCK, SG, NST, true, PROJ>(u, g, l, a.par, (a.t0 + blockIdx.y) * vsh + off, (T)a.omega,
                                                        a.hits, a.track, pre, post, (typename S::V *)staged_smem,
                                                        a.status);
    if (a.track) {
        // the reduction's scratch reuses the staging buffer: it has no static shared
        // memory, so 32-site blocks fit 12 to an SM; every thread is done with its
        // staged links after the barrier
        __syncthreads();
        auto *sh = reinterpret_cast<double(*)[BLOCK / 32]>(staged_smem);
        int &last = *reinterpret_cast<int *>(staged_smem + 2 * (BLOCK / 32) * sizeof(double));
        fused_reduce<BLOCK>(a, pre, post, sh, last);
    }
}

// projectSU3 on entries [begin, begin + count) of each of nblk SoA blocks
template <class S>
__global__ void k_reunit_fast(typename S::V *__restrict__ base, uint32_t stride, uint32_t nblk, uint32_t begin,
                              uint32_t count, const unsigned *stop, unsigned *status) {
    if (stop && *(volatile const unsigned *)stop) return;
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    if (j >= count || k >= nblk) return;
    uint32_t i = begin + j;
    typename S::V *p = base + (size_t)k * S::NS * stride + i;
    Mt<typename S::T> m;
    S::load(p, stride, m);
    if (!fproject(m)) atomicOr(status, GFC_STATUS_PROJECT_FAIL);
    S::store(p, stride, m);
}

// FP64 full SoA -> FP32 two-row SoA (nblk blocks of [9][stride] -> [3][stride])
__global__ void k_to_f32(const double2 *__restrict__ src, float4 *__restrict__ dst, uint32_t stride, uint32_t nblk) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    if (i >= stride || k >= nblk) return;
    const double2 *p = src + (size_t)k * 9 * stride + i;
    float4 *q = dst + (size_t)k * 3 * stride + i;
    double2 e[6];
#pragma unroll
    for (int c = 0; c < 6; c++) e[c] = p[(size_t)c * stride];
    q[0] = make_float4((float)e[0].x, (float)e[0].y, (float)e[1].x, (float)e[1].y);
    q[stride] = make_float4((float)e[2].x, (float)e[2].y, (float)e[3].x, (float)e[3].y);
    q[2 * (size_t)stride] = make_float4((float)e[4].x, (float)e[4].y, (float)e[5].x, (float)e[5].y);
}

// FP32 two-row SoA -> FP64 full SoA, row 2 rebuilt and the result projected in FP64
__global__ void k_to_f64(const float4 *__restrict__ src, double2 *__restrict__ dst, uint32_t stride, uint32_t nblk) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    if (i >= stride || k >= nblk) return;
    const float4 *p = src + (size_t)k * 3 * stride + i;
    float4 a = p[0], b = p[stride], c = p[2 * (size_t)stride];
    Mt<double> m;
    m.e[0] = make_double2(a.x, a.y);
    m.e[1] = make_double2(a.z, a.w);
    m.e[2] = make_double2(b.x, b.y);
    m.e[3] = make_double2(b.z, b.w);
    m.e[4] = make_double2(c.x, c.y);
    m.e[5] = make_double2(c.z, c.w);
    if (!fproject(m)) fidentity(m);
    double2 *q = dst + (size_t)k * 9 * stride + i;
#pragma unroll
    for (int e = 0; e < 9; e++) q[(size_t)e * stride] = m.e[e];
}

// FP64 full SoA ([9][stride] per block) -> FP64 two-row SoA ([6][stride])
__global__ void k_pack2(const double2 *__restrict__ src, double2 *__restrict__ dst, uint32_t stride, uint32_t nblk) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    if (i >= stride || k >= nblk) return;
    const double2 *p = src + (size_t)k * 9 * stride + i;
    double2 *q = dst + (size_t)k * 6 * stride + i;
#pragma unroll
    for (int e = 0; e < 6; e++) q[(size_t)e * stride] = p[(size_t)e * stride];
}

// FP64 two-row -> full, row 2 = conj(row0 x row1)
__global__ void k_unpack2(const double2 *__restrict__ src, double2 *__restrict__ dst, uint32_t stride, uint32_t nblk) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    if (i >= stride || k >= nblk) return;
    Mt<double> m;
    S64R::load(src + (size_t)k * 6 * stride + i, stride, m);
    S64::store(dst + (size_t)k * 9 * stride + i, stride, m);
}

// Slice-blocked sweeping: after a round, e2 after s half-sweeps is
// sum_t post[s-1][t] + pre[s][t] from the per-slice ring.  Summed in slice order
// (deterministic).  Sets stop = 0x40000000 | s at the first s with e2 <= tol.
__global__ void k_round_check(const double *__restrict__ ring, int ring_n, int nt, int s_lo, int s_hi,
                              double *__restrict__ hist, int hist_n, double tol_sum, unsigned *stop,
                              unsigned *status) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (*(volatile unsigned *)stop) return;
    for (int s = s_lo; s <= s_hi; s++) {
        const double *po = ring + (size_t)((s - 1) % ring_n) * nt * 2;
        const double *pr = ring + (size_t)(s % ring_n) * nt * 2;
        double a = 0.0, b = 0.0;
        for (int t = 0; t < nt; t++) {
            a += pr[2 * t];
            b += po[2 * t + 1];
        }
        if (s < hist_n) hist[2 * s] = a;
        if (s - 1 < hist_n) hist[2 * (s - 1) + 1] = b;
        double e2 = a + b;
        if (!(e2 == e2)) {
            atomicOr(status, GFC_STATUS_NAN);
            *stop = 0x80000000u | (unsigned)s;
            return;
        }
        if (e2 <= tol_sum) {
            *stop = 0x40000000u | (unsigned)s;
            return;
        }
    }
}

__global__ void k_identity32(float4 *__restrict__ g, uint32_t stride, uint32_t nblk) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    if (i >= stride || k >= nblk) return;
    float4 *q = g + (size_t)k * 3 * stride + i;
    q[0] = make_float4(1.f, 0.f, 0.f, 0.f);
    q[stride] = make_float4(0.f, 0.f, 0.f, 0.f);
    q[2 * (size_t)stride] = make_float4(1.f, 0.f, 0.f, 0.f);
}

// Rebuilds of the mixed fix (checkerboard layout; one thread per (parity, site)
// slot, grid.y = parity).
//
// G <- Proj(G32 G) in FP64, G32's two rows widened, completed and projected first
// (as k_to_f64 does): a warm start's G0, or the G accumulated by earlier rebuilds,
// composed with the transformation of the FP32 phase; with reset32 the FP32 G
// restarts from the identity (as k_identity32 sets it).
__global__ void k_compose_gt(float4 *__restrict__ g32, double2 *__restrict__ g, uint32_t stride, int reset32) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    if (i >= stride) return;
    float4 *q = g32 + (size_t)k * 3 * stride + i;
    const float4 a = q[0], b = q[stride], cc = q[2 * (size_t)stride];
    Mt<double> m1, m0, r;
    m1.e[0] = make_double2(a.x, a.y);
    m1.e[1] = make_double2(a.z, a.w);
    m1.e[2] = make_double2(b.x, b.y);
    m1.e[3] = make_double2(b.z, b.w);
    m1.e[4] = make_double2(cc.x, cc.y);
    m1.e[5] = make_double2(cc.z, cc.w);
    if (!fproject(m1)) fidentity(m1);
    const size_t o = (size_t)k * 9 * stride + i;
    S64::load(g + o, stride, m0);
    fprod_left<S64, double>(m1, m0, r);
    if (!fproject(r)) fidentity(r);
    S64::store(g + o, stride, r);
    if (reset32) {
        q[0] = make_float4(1.f, 0.f, 0.f, 0.f);
        q[stride] = make_float4(0.f, 0.f, 0.f, 0.f);
        q[2 * (size_t)stride] = make_float4(1.f, 0.f, 0.f, 0.f);
    }
}

// rows 0 and 1 of o into two-row storage (FP32: rounded to nearest)
__device__ __forceinline__ void store_rows01(float4 *__restrict__ p, size_t st, const Mt<double> &o) {
    p[0] = make_float4((float)o.e[0].x, (float)o.e[0].y, (float)o.e[1].x, (float)o.e[1].y);
    p[st] = make_float4((float)o.e[2].x, (float)o.e[2].y, (float)o.e[3].x, (float)o.e[3].y);
    p[2 * st] = make_float4((float)o.e[4].x, (float)o.e[4].y, (float)o.e[5].x, (float)o.e[5].y);
}
__device__ __forceinline__ void store_rows01(double2 *__restrict__ p, size_t st, const Mt<double> &o) {
#pragma unroll
    for (int c = 0; c < 6; c++) p[(size_t)c * st] = o.e[c];
}

// Spatial links from the FP64 start: U_d(x) = G(x) U0_d(x) G(x+d)^dagger (FMA
// arithmetic), written straight into the two-row storage S of the next phase (FP32
// for a rebuild of the FP32 phase, FP64 at the switch to the refinement).
template <class S>
__global__ void __launch_bounds__(128) k_regauge(const double2 *__restrict__ u0, const double2 *__restrict__ g,
                                                 typename S::V *__restrict__ out, Lat l) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const int par = blockIdx.y;
    if (i >= l.vh) return;
    const Coord c = coord_cb(l, par, i);
    Mt<double> gx, gy, uu, t, o;
    S64::load(g + gidx(l, par, 0, i), l.vh, gx);
#pragma unroll 1
    for (int d = 0; d < 3; d++) {
        S64::load(g + gidx(l, par ^ 1, 0, fwd_L(l, c, d) >> 1), l.vh, gy);
        S64::load(u0 + uidx(l, d, par, 0, i), l.vh, uu);
        fprod_left<S64R, double>(gx, uu, t);   // rows 0, 1 of G(x) U0
        fprod_dag<S64R, double>(t, gy, o);     // rows 0, 1 of that times G(x+d)^dagger
        store_rows01(out + su_idx<S>(l, d, par, i), l.vh, o);
    }
}

// ------------------------------------------------------------------ host --
static int ensure_track_buffers(gfc_ctx *c, int hist_n) {
    const Lat &l = c->lat;
    uint32_t nbx = ((l.vs >> 1) + MIN_BLOCK - 1) / MIN_BLOCK;
    size_t need = (size_t)l.nt * nbx * 2 + (size_t)l.nt * 2;
    if (c->part_n < need) {
        cudaFree(c->part);
        c->part = nullptr;
        GFC_CHECK(cudaMalloc(&c->part, need * sizeof(double)));
        c->part_n = need;
    }
    if (c->hist_n < hist_n) {
        cudaFree(c->e2_hist);
        c->e2_hist = nullptr;
        GFC_CHECK(cudaMalloc(&c->e2_hist, (size_t)hist_n * 2 * sizeof(double)));
        c->hist_n = hist_n;
    }
    return GFC_OK;
}

// tickets and stop word live at the tail of the part buffer (as unsigned)
struct TrackPtrs {
    double *part, *slice;
    unsigned *tickets, *stop;
};
static TrackPtrs track_ptrs(gfc_ctx *c) {
    const Lat &l = c->lat;
    uint32_t nbx = ((l.vs >> 1) + MIN_BLOCK - 1) / MIN_BLOCK;
    TrackPtrs t;
    t.part = c->part;
    t.slice = c->part + (size_t)l.nt * nbx * 2;
    t.tickets = c->tickets;
    t.stop = c->tickets + (l.nt + 1);
    return t;
}

template <class S, int K>
static void launch_shape(dim3 grid, cudaStream_t st, typename S::V *u, typename S::V *g, const SweepArgs &a) {
    constexpr int B = kShapes[K].block;
    static_assert(B >= MIN_BLOCK, "block partial buffers are sized for MIN_BLOCK");
    grid.x = ((a.l.vs >> 1) + B - 1) / B;
    k_sweep_fast<S, B, kShapes[K].minb><<<grid, B, 0, st>>>(u, g, a);
}

template <class S>
static constexpr size_t staged_bytes(int block, int sg, int nst) {
    return (size_t)(nst + sg) * S::NS * block * sizeof(typename S::V);
}

template <class S, int K>
static void launch_staged(dim3 grid, cudaStream_t st, typename S::V *u, typename S::V *g, const SweepArgs &a) {
    constexpr SShape sh = kStaged[K];
    constexpr size_t bytes = staged_bytes<S>(sh.block, sh.sg, sh.nst);
    static_assert(bytes <= 227 * 1024, "staged tile exceeds shared memory");
    static_assert(sh.block >= MIN_BLOCK, "block partial buffers are sized for MIN_BLOCK");
    auto kern = k_sweep_staged<S, sh.block, sh.minb, (bool)sh.sg, sh.nst>;
    static std::atomic<unsigned long long> done{0};
    smem_attr_once(done, kern, bytes);
    grid.x = ((a.l.vs >> 1) + sh.block - 1) / sh.block;
    if constexpr ((std::is_same<S, S64R>::value || std::is_same<S, S32>::value) && sh.nst == 6) {
        if (a.proj) {
            auto kp = k_sweep_staged<S, sh.block, sh.minb, (bool)sh.sg, sh.nst, true>;
            static std::atomic<unsigned long long> done_p{0};
            smem_attr_once(done_p, kp, bytes);
            kp<<<grid, sh.block, bytes, st>>>(u, g, a);
            return;
        }
    }
    kern<<<grid, sh.block, bytes, st>>>(u, g, a);
}

// Whether a half-sweep launched with SweepArgs::proj projects the links it writes
// (the fully staged two-row shapes, FP64 and FP32); the others leave the links to a
// separate reunitarisation pass.
template <class S>
static bool links_fold_reunit(const gfc_ctx *c) {
    if constexpr (std::is_same<S, S64R>::value || std::is_same<S, S32>::value) {
        const int k = (std::is_same<S, S64R>::value ? c->shape_fast64 : c->shape_fast32) - kNumShapes;
        return k >= 0 && k < kNumStaged && kStaged[k].nst == 6;
    }
    return false;
}

template <class S>
static void dispatch_fast(int v, dim3 grid, cudaStream_t st, typename S::V *u, typename S::V *g,
                          const SweepArgs &a) {
    if constexpr (S::ROWS01_ONLY) {
        switch (v - kNumShapes) {
            case 0: return launch_staged<S, 0>(grid, st, u, g, a);
            case 1: return launch_staged<S, 1>(grid, st, u, g, a);
            case 2: return launch_staged<S, 2>(grid, st, u, g, a);
            case 3: return launch_staged<S, 3>(grid, st, u, g, a);
            case 4: return launch_staged<S, 4>(grid, st, u, g, a);
            case 5: return launch_staged<S, 5>(grid, st, u, g, a);
            case 6: return launch_staged<S, 6>(grid, st, u, g, a);
            case 7: return launch_staged<S, 7>(grid, st, u, g, a);
            case 8: return launch_staged<S, 8>(grid, st, u, g, a);
            default: break;
        }
    } else if (v >= kNumShapes) {
        v = 1;   // full 3x3 storage has no staged form
    }
    switch (v) {
        case 0: launch_shape<S, 0>(grid, st, u, g, a); break;
        case 1: launch_shape<S, 1>(grid, st, u, g, a); break;
        case 2: launch_shape<S, 2>(grid, st, u, g, a); break;
        case 3: launch_shape<S, 3>(grid, st, u, g, a); break;
        case 4: launch_shape<S, 4>(grid, st, u, g, a); break;
        case 5: launch_shape<S, 5>(grid, st, u, g, a); break;
        case 6: launch_shape<S, 6>(grid, st, u, g, a); break;
        case 7: launch_shape<S, 7>(grid, st, u, g, a); break;
        default: launch_shape<S, 8>(grid, st, u, g, a); break;
    }
}

// One half-sweep of timeslices [t0, t0 + nsl) (all slices by default).
template <class S>
static void launch_fast(gfc_ctx *c, typename S::V *u, typename S::V *g, int sweep, double omega, unsigned hits,
                        int track, unsigned *stop, double tol_sum, int t0 = 0, int nsl = -1, int test = 1,
                        int proj = 0) {
    const Lat &l = c->lat;
    TrackPtrs tp = track_ptrs(c);
    SweepArgs a{};
    a.l = l;
    a.par = sweep & 1;
    a.omega = omega;
    a.hits = hits;
    a.track = track;
    a.t0 = t0;
    a.part = tp.part;
    a.tickets = tp.tickets;
    a.slice = tp.slice;
    a.ring = c->ring;
    a.ring_n = c->ring_n;
    a.hist = c->e2_hist;
    a.sweep = sweep;
    a.hist_n = c->hist_n;
    a.stop = stop;
    a.tol_sum = tol_sum;
    a.test = test;
    a.status = c->dstatus;
    a.proj = proj;
    const int v = sizeof(typename S::T) == 8 ? c->shape_fast64 : c->shape_fast32;
    dispatch_fast<S>(v, dim3(0, nsl < 0 ? l.nt : nsl), c->s, u, g, a);
    c->launches++;
}

// The fast FP64 sweeps keep links and G as two stored rows (1344 B instead of 2016 B
// of traffic per site-update); the full-matrix fields u, g remain the canonical
// state that everything else reads.
static int ensure_2row(gfc_ctx *c) {
    const Lat &l = c->lat;
    if (!c->u64r) GFC_CHECK(cudaMalloc(&c->u64r, (size_t)3 * l.npar * l.vh * 6 * sizeof(double2)));
    if (!c->g64r) GFC_CHECK(cudaMalloc(&c->g64r, (size_t)l.npar * l.vh * 6 * sizeof(double2)));
    return GFC_OK;
}
static void pack_2row(gfc_ctx *c) {
    const Lat &l = c->lat;
    dim3 gu((l.vh + 255) / 256, 3 * l.npar), gg((l.vh + 255) / 256, l.npar);
    k_pack2<<<gu, 256, 0, c->s>>>(c->u, c->u64r, l.vh, 3 * l.npar);
    k_pack2<<<gg, 256, 0, c->s>>>(c->g, c->g64r, l.vh, l.npar);
    c->launches += 2;
}
static void unpack_2row(gfc_ctx *c) {
    const Lat &l = c->lat;
    dim3 gu((l.vh + 255) / 256, 3 * l.npar), gg((l.vh + 255) / 256, l.npar);
    k_unpack2<<<gu, 256, 0, c->s>>>(c->u64r, c->u, l.vh, 3 * l.npar);
    k_unpack2<<<gg, 256, 0, c->s>>>(c->g64r, c->g, l.vh, l.npar);
    c->launches += 2;
}

// launchers over nblk SoA blocks of `stride` matrices (used by the batch engine)
void launch_to_f32(const double2 *src, float4 *dst, uint32_t stride, uint32_t nblk, cudaStream_t s) {
    k_to_f32<<<dim3((stride + 255) / 256, nblk), 256, 0, s>>>(src, dst, stride, nblk);
}
void launch_identity32(float4 *g, uint32_t stride, uint32_t nblk, cudaStream_t s) {
    k_identity32<<<dim3((stride + 255) / 256, nblk), 256, 0, s>>>(g, stride, nblk);
}
void launch_pack2(const double2 *src, double2 *dst, uint32_t stride, uint32_t nblk, cudaStream_t s) {
    k_pack2<<<dim3((stride + 255) / 256, nblk), 256, 0, s>>>(src, dst, stride, nblk);
}
void launch_unpack2(const double2 *src, double2 *dst, uint32_t stride, uint32_t nblk, cudaStream_t s) {
    k_unpack2<<<dim3((stride + 255) / 256, nblk), 256, 0, s>>>(src, dst, stride, nblk);
}

int halfsweeps_fast64(gfc_ctx *c, int first, int n, double omega, unsigned hits) {
    int rc = ensure_track_buffers(c, 1);
    if (!rc) rc = ensure_2row(c);
    if (rc) return rc;
    pack_2row(c);
    for (int k = 0; k < n; k++) launch_fast<S64R>(c, c->u64r, c->g64r, first + k, omega, hits, 0, nullptr, 0.0);
    unpack_2row(c);
    return GFC_OK;
}

// reunitarise the matrices of timeslices [t0, t0 + nsl) in nblk SoA blocks
template <class S>
static void launch_reunit(gfc_ctx *c, typename S::V *base, uint32_t nblk, unsigned *stop, int t0 = 0,
                          int nsl = -1) {
    const Lat &l = c->lat;
    const uint32_t vsh = l.vs >> 1;
    const uint32_t begin = (uint32_t)t0 * vsh, count = nsl < 0 ? l.vh : (uint32_t)nsl * vsh;
    dim3 grid((count + 255) / 256, nblk);
    k_reunit_fast<S><<<grid, 256, 0, c->s>>>(base, l.vh, nblk, begin, count, stop, c->dstatus);
    c->launches++;
}

static void print_res(int sweep, double res) { printf("Sweeps: %8d.\t residue: %3.2E \n", sweep, res); }

// ----------------------------------------------------------------- odd ns --
// Odd ns with the fast arithmetic (FP64 on two stored rows, lexicographic layout): a
// half-sweep is the four boundary-level launches of the exact path (the sequential
// sweep's order between every pair of sites that share a link, see
// k_sweep_exact_level), each thread taking a site of the half-sweep's parity
// (odd_parity_site) and updating it if it has the launch's level.  e2 is measured by
// a separate pass over the state a half-sweep leaves: a site's post-update w is not
// final while a later level updates a neighbour.
constexpr int LEX_BLOCK = 32;
__global__ void __launch_bounds__(LEX_BLOCK, 11) k_sweep_lex_fast(double2 *__restrict__ u, double2 *__restrict__ g,
                                                                 Lat l, int sweep, int level, double omega,
                                                                 unsigned hits, const unsigned *stop) {
    extern __shared__ __align__(16) unsigned char lex_stage[];
    if (stop && *(volatile const unsigned *)stop) return;
    uint32_t L;
    if (!odd_parity_site(l, sweep & 1, blockIdx.x * LEX_BLOCK + threadIdx.x, L)) return;
    const Coord c = coord_lex(l, L);
    const uint32_t e = (uint32_t)l.ns - 1;
    if ((int)(c.x == e) + (int)(c.y == e) + (int)(c.z == e) != level) return;
    double pre = 0.0, post = 0.0;
    fast_site_staged<S64R, LEX_BLOCK, false, 6, false>(u, g, l, 0, L, omega, hits, 0, pre, post,
                                                       (double2 *)lex_stage);
}

static void launch_halfsweep_lex_fast(gfc_ctx *c, int sweep, double omega, unsigned hits, const unsigned *stop) {
    const Lat &l = c->lat;
    constexpr size_t bytes = (size_t)6 * S64R::NS * LEX_BLOCK * sizeof(double2);
    static std::atomic<unsigned long long> done{0};
    smem_attr_once(done, k_sweep_lex_fast, bytes);
    const unsigned blocks = (unsigned)((l.v / 2 + 1 + LEX_BLOCK - 1) / LEX_BLOCK);
    for (int level = 0; level < 4; level++)
        k_sweep_lex_fast<<<blocks, LEX_BLOCK, bytes, c->s>>>(c->u64r, c->g64r, l, sweep, level, omega, hits, stop);
    c->launches += 4;
}

// e2 and theta partials (theta = e2 / 6 identically) per timeslice of the two-row
// lexicographic links: grid (nbx, nt), fixed summation order
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_e2_lex_fast(const double2 *__restrict__ u, Lat l,
                                                       double *__restrict__ part, const unsigned *stop) {
    if (stop && *(volatile const unsigned *)stop) return;
    __shared__ double sh[2][BLOCK / 32];
    const uint32_t t = blockIdx.y;
    double v[2] = {0.0, 0.0};
    for (uint32_t k = blockIdx.x * BLOCK + threadIdx.x; k < l.vs; k += gridDim.x * BLOCK) {
        const double e2 = measure_site<S64R, false>(u, l, 0, t * l.vs + k);
        v[0] += e2;
        v[1] += 0.5 * e2;   // Re Tr(div A div A^dagger) of the site
    }
    fblock_sum<BLOCK, 2>(v, sh);
    if (threadIdx.x == 0) {
        const size_t o = ((size_t)t * gridDim.x + blockIdx.x) * 2;
        part[o] = v[0];
        part[o + 1] = v[1];
    }
}

static void launch_e2_lex_fast(gfc_ctx *c, const unsigned *stop) {
    const Lat &l = c->lat;
    const int nbx = obs_blocks_per_slice(l);
    k_e2_lex_fast<128><<<dim3(nbx, l.nt), 128, 0, c->s>>>(c->u64r, l, c->part, stop);
    launch_finalize2(c->part, l, nbx, c->dres, c->s, stop);
    c->launches += 2;
}

// n half-sweeps from `first` on the two stored rows (packed before, unpacked after),
// for the reference's check schedule
int halfsweeps_odd_fast(gfc_ctx *c, int first, int n, double omega, unsigned hits) {
    int rc = ensure_2row(c);
    if (rc) return rc;
    pack_2row(c);
    for (int k = 0; k < n; k++) launch_halfsweep_lex_fast(c, first + k, omega, hits, nullptr);
    unpack_2row(c);
    return GFC_OK;
}

// Stop at the first half-sweep whose proxy is below the tolerance (the schedule of
// the exact path's every-half-sweep fix: measured at the end of each chunk of 32 while
// the tolerance is far, after every half-sweep near it; the test on the device).
int fix_every_sweep_odd_fast(gfc_ctx *c, const gfc_params *p, const gfc_options *o, gfc_report *r) {
    const Lat &l = c->lat;
    const double omega = (double)p->omega_OR;
    double e2 = 0.0, th = 0.0;
    int rc = gfc_ctx_e2(c, &e2, &th);
    if (rc) return rc;
    const int theta = p->gfix_proxy == GFC_PROXY_THETA;
    const double res0 = theta ? th : e2;
    r->initial_residue = res0;
    if (o->verbose) print_res(0, res0);
    GFC_CHECK(cudaEventRecord(c->ev_b, c->s));
    if (res0 <= p->tolerance) {
        GFC_CHECK(cudaEventRecord(c->ev_d, c->s));
        r->sweeps = 0;
        r->first_below_tol = 0;
        return 0;
    }
    if ((rc = ensure_2row(c))) return rc;
    pack_2row(c);
    unsigned *stop = c->tickets + (l.nt + 1);
    GFC_CHECK(cudaMemsetAsync(stop, 0, sizeof(unsigned), c->s));
    const int max = (int)p->max_sweeps_to_fix, period = (int)p->sweeps_to_reunitarization;
    unsigned hstop = 0;
    bool dense = o->dense_check != 0;
    int sweep = 0, k_a = -1;
    double res_a = 0.0;
    while (sweep < max) {
        int end = std::min(max, sweep + 32);
        if (period > 0) end = std::min(end, (sweep / period + 1) * period);
        for (; sweep < end; sweep++) {
            launch_halfsweep_lex_fast(c, sweep, omega, p->hits, stop);
            if (dense || sweep + 1 == end) {
                launch_e2_lex_fast(c, stop);
                launch_exact_check(c->dres, l, theta, p->tolerance, sweep + 1, stop, c->s);
                c->launches++;
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
        if (period > 0 && !(sweep % period)) {
            launch_reunit<S64R>(c, c->u64r, 3 * l.npar, stop);
            launch_reunit<S64R>(c, c->g64r, l.npar, stop);
        }
    }
    unpack_2row(c);
    GFC_CHECK(cudaEventRecord(c->ev_d, c->s));
    if (hstop) {
        sweep = (int)hstop;
        r->first_below_tol = sweep;
    }
    r->sweeps = sweep;
    r->site_updates = (long long)sweep * (l.v / 2);
    return hstop ? sweep : GFC_FIX_NOT_CONVERGED;
}

static int ensure_ring(gfc_ctx *c, int ring_n) {
    if (c->ring_n >= ring_n) return GFC_OK;
    cudaFree(c->ring);
    c->ring = nullptr;
    GFC_CHECK(cudaMalloc(&c->ring, (size_t)ring_n * c->lat.nt * 2 * sizeof(double)));
    c->ring_n = ring_n;
    return GFC_OK;
}

// Slice-blocked round: half-sweeps [sweep, kend) applied to one group of G
// timeslices after another.  Timeslices share no link during the sweeps, so a
// group can run several half-sweeps while its links and G stay in L2 (kernel
// boundaries order the half-sweeps); e2 partials go to the per-slice ring.
template <class S>
static void sweep_round(gfc_ctx *c, typename S::V *u, typename S::V *g, int sweep, int kend, int G, double omega,
                        unsigned hits, unsigned reunit, unsigned *stop) {
    const Lat &l = c->lat;
    for (int g0 = 0; g0 < l.nt; g0 += G) {
        const int gn = std::min(G, l.nt - g0);
        for (int k = sweep; k < kend; k++) {
            launch_fast<S>(c, u, g, k, omega, hits, 2, stop, 0.0, g0, gn);
            if (reunit && !((k + 1) % reunit)) {
                launch_reunit<S>(c, u, 3 * l.npar, stop, g0, gn);
                launch_reunit<S>(c, g, l.npar, stop, g0, gn);
            }
        }
    }
}


static int initial_proxy(gfc_ctx *c, const gfc_params *p, double *e2, double *res) {
    double th;
    int rc = gfc_ctx_e2(c, e2, &th);
    if (rc) return rc;
    *res = p->gfix_proxy == GFC_PROXY_THETA ? th : *e2;
    return GFC_OK;
}

static int read_stop(gfc_ctx *c, const unsigned *stop, unsigned *h) {
    GFC_CHECK(cudaMemcpyAsync(c->hres + 16, stop, sizeof(unsigned), cudaMemcpyDeviceToHost, c->s));
    GFC_CHECK(cudaStreamSynchronize(c->s));
    GFC_CHECK(cudaGetLastError());
    memcpy(h, c->hres + 16, sizeof *h);
    return GFC_OK;
}

// Run fused-e2 half-sweeps of storage S from sweep index sweep0 until the tracked
// e2 <= tol_e2, max_sweeps is reached, or an error.  *done = half-sweeps completed
// (global index), *first_below = the first half-sweep count whose e2 was seen
// <= tol (-1 if none).  Unblocked, the kernel that sees it stops the stream (one
// half-sweep late); slice-blocked, the round in progress is completed.
template <class S>
static int run_until(gfc_ctx *c, typename S::V *u, typename S::V *g, int sweep0, int max_sweeps, double tol_e2,
                     double omega, unsigned hits, unsigned reunit, int dense_check, int *done, int *first_below) {
    const Lat &l = c->lat;
    int rc = ensure_track_buffers(c, max_sweeps + 2);
    if (rc) return rc;
    TrackPtrs tp = track_ptrs(c);
    GFC_CHECK(cudaMemsetAsync(tp.tickets, 0, (l.nt + 2) * sizeof(unsigned), c->s));
    const double tol_sum = tol_e2 * (double)l.v;
    const int bs = sizeof(typename S::T) == 8 ? c->blk64_slices : c->blk32_slices;
    const int bk = sizeof(typename S::T) == 8 ? c->blk64_sweeps : c->blk32_sweeps;
    const int G = bs > 0 ? std::min(bs, l.nt) : l.nt;
    const int K = std::max(1, bk);
    int sweep = sweep0;
    unsigned hstop = 0;
    *first_below = -1;
    if (G >= l.nt && K == 1) {
        // e2 after half-sweep k needs the fused sums of half-sweeps k and k + 1.
        // While the tolerance is far (by the last measured value and the rate
        // between the last two measurements) only the last pair of each chunk of 32
        // is measured; from then on every half-sweep is, so the stop is still at the
        // first half-sweep whose e2 is below the tolerance.  The measuring costs
        // about a sixth of a half-sweep's time.
        const int chunk = 32;
        bool dense = dense_check != 0;
        bool prev_tracked = false;
        int k_a = -1;
        double e2_a = 0.0;
        while (sweep < max_sweeps) {
            const int end = std::min(max_sweeps, sweep + chunk);
            const int first_tracked = dense ? sweep : std::max(sweep, end - 2);
            for (; sweep < end; sweep++) {
                const int tr = sweep >= first_tracked;
                // a reunitarisation due after this half-sweep: the links it writes
                // (every spatial link) are projected by the sweep itself where the
                // shape can, leaving G's pass alone
                const bool ru = reunit && !((sweep + 1) % reunit);
                const bool fold = ru && links_fold_reunit<S>(c);
                launch_fast<S>(c, u, g, sweep, omega, hits, tr, tp.stop, tol_sum, 0, -1, tr && prev_tracked, fold);
                prev_tracked = tr;
                if (ru) {
                    if (!fold) launch_reunit<S>(c, u, 3 * l.npar, tp.stop);
                    launch_reunit<S>(c, g, l.npar, tp.stop);
                }
            }
            const int k = end - 2;   // e2 after half-sweep k is known from this chunk's pair
            const bool measured = !dense && k >= first_tracked && k + 1 < c->hist_n;
            if (measured)
                GFC_CHECK(cudaMemcpyAsync(c->hres + 20, c->e2_hist + 2 * k + 1, 2 * sizeof(double),
                                          cudaMemcpyDeviceToHost, c->s));
            if ((rc = read_stop(c, tp.stop, &hstop))) return rc;
            if (hstop) break;
            if (measured) {
                const double e2 = (c->hres[20] + c->hres[21]) / (double)l.v;   // post(k) + pre(k + 1)
                if (!(e2 == e2)) break;   // NaN: the status word has it; stop sweeping
                if (e2 <= 1e3 * tol_e2) {
                    dense = true;
                } else if (k_a >= 0 && e2 < e2_a) {
                    const double rate = pow(e2 / e2_a, 1.0 / (double)(k - k_a));
                    if (e2 * pow(rate, 2.0 * chunk) <= 10.0 * tol_e2) dense = true;
                }
                k_a = k;
                e2_a = e2;
            }
        }
        if (hstop & 0x80000000u) {
            set_error("NaN in the gauge functional at half-sweep %u", hstop & 0x7fffffffu);
            return GFC_ERR_NUMERIC;
        }
        if (hstop) {
            *done = (int)hstop;
            *first_below = (int)hstop - 1;
        } else {
            *done = sweep;
        }
        return GFC_OK;
    }
    if ((rc = ensure_ring(c, K + 2))) return rc;
    int s_lo = sweep0 + 1;
    while (sweep < max_sweeps) {
        const int kend = std::min(max_sweeps, sweep + K);
        sweep_round<S>(c, u, g, sweep, kend, G, omega, hits, reunit, tp.stop);
        if (kend - 1 >= s_lo) {
            k_round_check<<<1, 32, 0, c->s>>>(c->ring, c->ring_n, l.nt, s_lo, kend - 1, c->e2_hist, c->hist_n,
                                             tol_sum, tp.stop, c->dstatus);
            c->launches++;
        }
        s_lo = kend;
        sweep = kend;
        if ((rc = read_stop(c, tp.stop, &hstop))) return rc;
        if (hstop) break;
    }
    if (hstop & 0x80000000u) {
        set_error("NaN in the gauge functional at half-sweep %u", hstop & 0x3fffffffu);
        return GFC_ERR_NUMERIC;
    }
    *done = sweep;
    if (hstop) *first_below = (int)(hstop & 0x3fffffffu);
    return GFC_OK;
}

// The fused stop sees e2 after half-sweep k inside half-sweep k + 1, so the state a
// fast fix returns is one over-relaxed half-sweep later.  Its e2 is almost always
// lower still, but over-relaxation can raise e2 for a half-sweep (most visibly on
// tiny lattices).  Measure the returned state exactly (full FP64 fields in c->u) and,
// while it is above the tolerance, keep sweeping with e2 measured after every
// half-sweep.  *done is the global half-sweep count, updated.
template <class S>
static int settle(gfc_ctx *c, typename S::V *u, typename S::V *g, const gfc_params *p, double tol_e2,
                  unsigned reunit, int *done) {
    constexpr bool TWO_ROW = S::ROWS01_ONLY;
    for (int attempt = 0; attempt < 16 && *done < (int)p->max_sweeps_to_fix; attempt++) {
        double e2 = 0.0, th = 0.0;
        int rc = gfc_ctx_e2(c, &e2, &th);
        if (rc) return rc;
        if (e2 <= tol_e2) return GFC_OK;
        int more = 0, below = -1;
        rc = run_until<S>(c, u, g, *done, (int)p->max_sweeps_to_fix, tol_e2, (double)p->omega_OR, p->hits, reunit, 1,
                          &more, &below);
        if (rc) return rc;
        *done = more;
        if (TWO_ROW) unpack_2row(c);
        if (below < 0) return GFC_OK;   // the sweep budget ran out
    }
    return GFC_OK;
}

int fix_every_sweep(gfc_ctx *c, const gfc_params *p, const gfc_options *o, gfc_report *r) {
    const Lat &l = c->lat;
    double e2, res;
    int rc = initial_proxy(c, p, &e2, &res);
    if (rc) return rc;
    r->initial_residue = res;
    if (o->verbose) print_res(0, res);
    GFC_CHECK(cudaEventRecord(c->ev_b, c->s));
    if (res <= p->tolerance) {
        r->sweeps = 0;
        r->first_below_tol = 0;
        GFC_CHECK(cudaEventRecord(c->ev_d, c->s));
        return 0;
    }
    // theta = e2 / 6 identically (gauge_fixing.c:341-442)
    double tol_e2 = p->gfix_proxy == GFC_PROXY_THETA ? 6.0 * p->tolerance : p->tolerance;
    int done = 0, below = -1;
    if (o->precision == GFC_PREC_FP64_FULL) {
        // plain FP64: full 3x3 storage, same fast arithmetic
        rc = run_until<S64>(c, c->u, c->g, 0, (int)p->max_sweeps_to_fix, tol_e2, (double)p->omega_OR, p->hits,
                            p->sweeps_to_reunitarization, o->dense_check, &done, &below);
        if (rc) return rc;
        if (below >= 0 && (rc = settle<S64>(c, c->u, c->g, p, tol_e2, p->sweeps_to_reunitarization, &done)))
            return rc;
    } else {
        if ((rc = ensure_2row(c))) return rc;
        pack_2row(c);
        rc = run_until<S64R>(c, c->u64r, c->g64r, 0, (int)p->max_sweeps_to_fix, tol_e2, (double)p->omega_OR,
                             p->hits, p->sweeps_to_reunitarization, o->dense_check, &done, &below);
        if (rc) return rc;
        unpack_2row(c);
        if (below >= 0 &&
            (rc = settle<S64R>(c, c->u64r, c->g64r, p, tol_e2, p->sweeps_to_reunitarization, &done)))
            return rc;
    }
    GFC_CHECK(cudaEventRecord(c->ev_d, c->s));
    r->sweeps = done;
    r->first_below_tol = below;
    r->site_updates = (long long)done * l.vh;
    return below >= 0 ? done : GFC_FIX_NOT_CONVERGED;
}

int fix_mixed(gfc_ctx *c, const gfc_params *p, const gfc_options *o, gfc_report *r) {
    const Lat &l = c->lat;
    if (!c->u32 || !c->g32 || !c->u0) {
        set_error("context was created without GFC_CTX_MIXED");
        return GFC_ERR_STATE;
    }
    double e2, res;
    int rc = initial_proxy(c, p, &e2, &res);
    if (rc) return rc;
    r->initial_residue = res;
    if (o->verbose) print_res(0, res);
    GFC_CHECK(cudaEventRecord(c->ev_b, c->s));
    if (res <= p->tolerance) {
        r->sweeps = 0;
        r->first_below_tol = 0;
        GFC_CHECK(cudaEventRecord(c->ev_d, c->s));
        return 0;
    }
    const double tol_e2 = p->gfix_proxy == GFC_PROXY_THETA ? 6.0 * p->tolerance : p->tolerance;
    const double sw = std::max(o->switch_e2 > 0 ? o->switch_e2 : 1e-9, tol_e2);
    // the FP64 links of the start, re-gauged by the rebuilds and at the switch: the
    // links as uploaded, before G0 was applied, for a warm start (kept in u0); else
    // the FP64 links themselves, which nothing writes until the switch
    const double2 *U0 = o->warm_start ? c->u0 : c->u;
    const dim3 gu((l.vh + 255) / 256, 3 * l.npar), gg((l.vh + 255) / 256, l.npar), gs((l.vh + 127) / 128, l.npar);
    const int maxs = (int)p->max_sweeps_to_fix, K = o->fp32_refresh > 0 ? o->fp32_refresh : 0;
    int done = 0, below = -1;
    bool rebuilt = false;
    k_to_f32<<<gu, 256, 0, c->s>>>(c->u, (float4 *)c->u32, l.vh, 3 * l.npar);
    k_identity32<<<gg, 256, 0, c->s>>>((float4 *)c->g32, l.vh, l.npar);
    c->launches += 2;
    // FP32 bulk, in pieces of fp32_refresh half-sweeps when refreshing.  Without
    // refreshing, the FP32 links and G are reunitarised every min(reunit, 50)
    // half-sweeps; a refresh rebuilds them from the FP64 start and a projected FP64 G,
    // which takes the reunitarisation's place.
    const unsigned reunit32 = K ? 0u : std::min<unsigned>(p->sweeps_to_reunitarization, 50u);
    for (;;) {
        const int lim = K ? std::min(maxs, done + K) : maxs;
        int d = done;
        rc = run_until<S32>(c, (float4 *)c->u32, (float4 *)c->g32, done, lim, sw, (double)p->omega_OR, p->hits,
                            reunit32, o->dense_check, &d, &below);
        if (rc) return rc;
        done = d;
        if (below >= 0 || !K || done >= maxs) break;
        // refresh: G = G32 G in FP64 (projected) and the FP32 G back to the identity,
        // then the FP32 links rounded from G U0 G^dagger computed in FP64
        k_compose_gt<<<gg, 256, 0, c->s>>>((float4 *)c->g32, c->g, l.vh, 1);
        k_regauge<S32><<<gs, 128, 0, c->s>>>(U0, c->g, (float4 *)c->u32, l);
        c->launches += 2;
        rebuilt = true;
    }
    r->sweeps_fp32 = done;
    if (below < 0) {
        // the FP64 links follow G at the last refresh (the state the FP64 fields hold)
        if (rebuilt) {
            if (o->warm_start)
                launch_apply_gt_spatial(c->u, c->u0, c->g, l, c->s);
            else
                launch_apply_gt(c->u, c->ut, c->g, l, 0, c->s);   // in place, spatial links only
            c->launches++;
        }
        r->sweeps = done;
        GFC_CHECK(cudaEventRecord(c->ev_d, c->s));
        return GFC_FIX_NOT_CONVERGED;
    }
    // switch: G in FP64 (rebuilt and projected), U = G U0 G^dagger from the FP64 start,
    // both straight into the two-row storage of the refinement
    if ((rc = ensure_2row(c))) return rc;
    if (o->warm_start || K) {
        // G = G1 G0: G1 of the FP32 phase times the starting G0 (a warm start's, or
        // the one accumulated by the refreshes)
        k_compose_gt<<<gg, 256, 0, c->s>>>((float4 *)c->g32, c->g, l.vh, 0);
    } else {
        k_to_f64<<<gg, 256, 0, c->s>>>((const float4 *)c->g32, c->g, l.vh, l.npar);
    }
    k_regauge<S64R><<<gs, 128, 0, c->s>>>(U0, c->g, c->u64r, l);
    k_pack2<<<gg, 256, 0, c->s>>>(c->g, c->g64r, l.vh, l.npar);
    c->launches += 3;
    // FP64 refinement
    unsigned reunit64 = o->refine_reunit ? o->refine_reunit : p->sweeps_to_reunitarization;
    int done64 = 0;
    rc = run_until<S64R>(c, c->u64r, c->g64r, done, (int)p->max_sweeps_to_fix, tol_e2, (double)p->omega_OR,
                         p->hits, reunit64, o->dense_check, &done64, &below);
    if (rc) return rc;
    unpack_2row(c);
    if (below >= 0 && (rc = settle<S64R>(c, c->u64r, c->g64r, p, tol_e2, reunit64, &done64))) return rc;
    GFC_CHECK(cudaEventRecord(c->ev_d, c->s));
    r->sweeps = done64;
    r->first_below_tol = below;
    // site-updates in each precision
    r->site_updates = (long long)done64 * l.vh;
    return below >= 0 ? done64 : GFC_FIX_NOT_CONVERGED;
}

}  // namespace gfc

// ------------------------------------------------------------- autotuner --
// Times every compiled launch shape of the sweep kernels on the resident lattice
// and keeps the fastest per kernel.  The links are saved first and restored after
// (the timed half-sweeps change them), and G is reset to the identity.
// times (optional, length >= GFC_TUNE_SLOTS) receives seconds per half-sweep:
//   [0..4] exact shapes, [5..22] FP64 fast shapes (9 plain, then 9 staged), [23..40]
//   FP32 shapes, [41..44] FP64 slice blocking, [45..48] FP32 slice blocking (0: not timed).
using namespace gfc;

extern "C" int gfc_ctx_autotune(gfc_ctx *c, int which, double *times_out) {
    if (!c) return GFC_ERR_ARG;
    if (!c->has_links) return GFC_ERR_STATE;
    if (!which) which = 7;
    double times[GFC_TUNE_SLOTS] = {0.0};
    if (times_out)
        for (int k = 0; k < GFC_TUNE_SLOTS; k++) times_out[k] = 0.0;
    if (!c->lat.cb) return GFC_OK;   // odd ns: one kernel (boundary levels), nothing to choose
    GFC_CHECK(cudaSetDevice(c->dev));
    int rc = gfc_ctx_save_links(c);
    if (rc) return rc;
    const Lat &l = c->lat;
    const int n = 10;
    rc = ensure_track_buffers(c, 2 * n + 2);
    if (rc) return rc;
    TrackPtrs tp = track_ptrs(c);
    cudaEvent_t e0 = c->ev_a, e1 = c->ev_c;
    auto timed = [&](auto launch) -> double {
        for (int k = 0; k < 2; k++) launch(k);
        cudaEventRecord(e0, c->s);
        for (int k = 0; k < n; k++) launch(k);
        cudaEventRecord(e1, c->s);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        return ms * 1e-3 / n;
    };
    auto args_for = [&](int sweep) {
        SweepArgs a{};
        a.l = l;
        a.par = sweep & 1;
        a.omega = 1.95;
        a.hits = 2;
        a.track = 0;   // as most launches of a fix: e2 is measured on a few of them
        a.t0 = 0;
        a.ring = c->ring;
        a.ring_n = c->ring_n;
        a.part = tp.part;
        a.tickets = tp.tickets;
        a.slice = tp.slice;
        a.hist = c->e2_hist;
        a.sweep = sweep;
        a.hist_n = c->hist_n;
        a.stop = nullptr;
        a.tol_sum = 0.0;
        a.status = c->dstatus;
        return a;
    };
    if (which & 1) {
        double best = 1e30;
        for (int s = 0; s < kNE && s < exact_num_shapes(); s++) {
            double t = timed([&](int k) { launch_sweep_exact(c->u, c->g, l, k, 1.95, 2, c->s, s); });
            times[s] = t;
            if (t < best) {
                best = t;
                c->shape_exact = s;
            }
        }
    }
    if (which & 2) {
        if ((rc = ensure_2row(c))) return rc;
        pack_2row(c);
        double best = 1e30;
        for (int v = 0; v < kNumAll; v++) {
            double t = timed(
                [&](int k) { dispatch_fast<S64R>(v, dim3(0, l.nt), c->s, c->u64r, c->g64r, args_for(k)); });
            times[kNE + v] = t;
            if (t < best) {
                best = t;
                c->shape_fast64 = v;
            }
        }
    }
    if ((which & 4) && c->u32 && c->g32) {
        dim3 gu((l.vh + 255) / 256, 3 * l.npar), gg((l.vh + 255) / 256, l.npar);
        k_to_f32<<<gu, 256, 0, c->s>>>(c->u, (float4 *)c->u32, l.vh, 3 * l.npar);
        k_identity32<<<gg, 256, 0, c->s>>>((float4 *)c->g32, l.vh, l.npar);
        double best = 1e30;
        for (int v = 0; v < kNumAll; v++) {
            double t = timed([&](int k) {
                dispatch_fast<S32>(v, dim3(0, l.nt), c->s, (float4 *)c->u32, (float4 *)c->g32, args_for(k));
            });
            times[kNE + kNumAll + v] = t;
            if (t < best) {
                best = t;
                c->shape_fast32 = v;
            }
        }
    }
    // slice blocking: candidate group sizes from an L2 budget, K half-sweeps per visit
    GFC_CHECK(cudaMemsetAsync(tp.stop, 0, sizeof(unsigned), c->s));
    auto tune_blocking = [&](auto tag, auto *u, auto *g, int bytes_per_matrix, int &best_g, int &best_k,
                             double base_time, double *slot) -> int {
        using S = decltype(tag);
        const double slice_bytes = (double)l.vs * 4.0 * bytes_per_matrix;   // 3 links + G per site
        const int gmax = std::max(1, (int)(96.0e6 / slice_bytes));
        int cands[3] = {std::max(1, gmax / 2), gmax, 2 * gmax};
        double best = base_time;
        best_g = 0;
        best_k = 1;
        int slot_i = 0;
        for (int ci = 0; ci < 3; ci++) {
            const int G = cands[ci];
            if (G >= l.nt || (ci > 0 && G == cands[ci - 1])) continue;
            for (int K : {4, 8}) {
                int e = ensure_ring(c, K + 2);
                if (e) return e;
                sweep_round<S>(c, u, g, 0, K, G, 1.95, 2, 0, tp.stop);   // warm
                cudaEventRecord(e0, c->s);
                sweep_round<S>(c, u, g, K, 2 * K, G, 1.95, 2, 0, tp.stop);
                cudaEventRecord(e1, c->s);
                cudaEventSynchronize(e1);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                const double t = ms * 1e-3 / K;
                if (slot && slot_i < 4) slot[slot_i++] = t;
                if (t < best) {
                    best = t;
                    best_g = G;
                    best_k = K;
                }
            }
        }
        return GFC_OK;
    };
    if (which & 2) {
        double base = 1e30;
        for (int v = 0; v < kNumAll; v++)
            if (times[kNE + v] > 0 && times[kNE + v] < base) base = times[kNE + v];
        rc = tune_blocking(S64R{}, c->u64r, c->g64r, 96, c->blk64_slices, c->blk64_sweeps, base,
                           times + kNE + 2 * kNumAll);
        if (rc) return rc;
    }
    if ((which & 4) && c->u32 && c->g32) {
        double base = 1e30;
        for (int v = 0; v < kNumAll; v++)
            if (times[kNE + kNumAll + v] > 0 && times[kNE + kNumAll + v] < base) base = times[kNE + kNumAll + v];
        rc = tune_blocking(S32{}, (float4 *)c->u32, (float4 *)c->g32, 48, c->blk32_slices, c->blk32_sweeps, base,
                           times + kNE + 4 + 2 * kNumAll);
        if (rc) return rc;
    }
    GFC_CHECK(cudaGetLastError());
    rc = gfc_ctx_restore_links(c);
    if (rc) return rc;
    launch_identity(c->g, l, c->s);
    GFC_CHECK(cudaStreamSynchronize(c->s));
    c->tuned = 1;
    if (times_out)
        for (int k = 0; k < GFC_TUNE_SLOTS; k++) times_out[k] = times[k];
    return GFC_OK;
}

extern "C" int gfc_ctx_set_blocking(gfc_ctx *c, int precision_bits, int slices, int sweeps) {
    if (!c || slices < 0 || sweeps < 1) return GFC_ERR_ARG;
    if (precision_bits & 2) {
        c->blk64_slices = slices;
        c->blk64_sweeps = sweeps;
    }
    if (precision_bits & 4) {
        c->blk32_slices = slices;
        c->blk32_sweeps = sweeps;
    }
    return GFC_OK;
}

extern "C" int gfc_ctx_get_blocking(const gfc_ctx *c, int *s64, int *k64, int *s32, int *k32) {
    if (!c) return GFC_ERR_ARG;
    if (s64) *s64 = c->blk64_slices;
    if (k64) *k64 = c->blk64_sweeps;
    if (s32) *s32 = c->blk32_slices;
    if (k32) *k32 = c->blk32_sweeps;
    return GFC_OK;
}

extern "C" int gfc_ctx_get_shapes(const gfc_ctx *c, int *exact, int *fast64, int *fast32) {
    if (!c) return GFC_ERR_ARG;
    if (exact) *exact = c->shape_exact;
    if (fast64) *fast64 = c->shape_fast64;
    if (fast32) *fast32 = c->shape_fast32;
    return GFC_OK;
}

extern "C" int gfc_ctx_set_shapes(gfc_ctx *c, int exact, int fast64, int fast32) {
    if (!c) return GFC_ERR_ARG;
    if (exact >= exact_num_shapes() || fast64 >= kNumAll || fast32 >= kNumAll) return GFC_ERR_ARG;
    if (exact >= 0) c->shape_exact = exact;
    if (fast64 >= 0) c->shape_fast64 = fast64;
    if (fast32 >= 0) c->shape_fast32 = fast32;
    return GFC_OK;
}
