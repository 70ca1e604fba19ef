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

namespace gfc {

template <typename T>
struct CT;
template <>
struct CT<double> {
    using t = double2;
};
template <>
struct CT<float> {
    using t = float2;
};

template <typename T>
struct Mt {
    typename CT<T>::t e[9];
};

template <typename C>
__device__ __forceinline__ C mkc(decltype(C::x) a, decltype(C::x) b) {
    C r;
    r.x = a;
    r.y = b;
    return r;
}
template <typename C>
__device__ __forceinline__ C fmul(C a, C b) {
    return mkc<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C>
__device__ __forceinline__ C fmul_conj(C a, C b) {  // a * conj(b)
    return mkc<C>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename C>
__device__ __forceinline__ C fadd(C a, C b) {
    return mkc<C>(a.x + b.x, a.y + b.y);
}
template <typename C>
__device__ __forceinline__ C fconj(C a) {
    return mkc<C>(a.x, -a.y);
}

__device__ __forceinline__ double frsqrt(double x) { return rsqrt(x); }
__device__ __forceinline__ float frsqrt(float x) { return rsqrtf(x); }

// conj(a x b)
template <typename C>
__device__ __forceinline__ void fcross_conj(const C *a, const C *b, C *o) {
    o[0] = fconj(fadd(fmul(a[1], b[2]), mkc<C>(-(a[2].x * b[1].x - a[2].y * b[1].y), -(a[2].x * b[1].y + a[2].y * b[1].x))));
    o[1] = fconj(fadd(fmul(a[2], b[0]), mkc<C>(-(a[0].x * b[2].x - a[0].y * b[2].y), -(a[0].x * b[2].y + a[0].y * b[2].x))));
    o[2] = fconj(fadd(fmul(a[0], b[1]), mkc<C>(-(a[1].x * b[0].x - a[1].y * b[0].y), -(a[1].x * b[0].y + a[1].y * b[0].x))));
}

template <typename T>
__device__ __forceinline__ void reconstruct_row2(Mt<T> &m) {
    fcross_conj(&m.e[0], &m.e[3], &m.e[6]);
}

// ---------------------------------------------------------------- storage --
struct S64 {
    using T = double;
    using V = double2;
    static constexpr int NS = 9;
    static constexpr int BYTES = 144;
    __device__ static void load(const V *__restrict__ p, size_t st, Mt<T> &m) {
#pragma unroll
        for (int c = 0; c < 9; c++) m.e[c] = p[(size_t)c * st];
    }
    __device__ static void load_rows01(const V *__restrict__ p, size_t st, Mt<T> &m) {
#pragma unroll
        for (int c = 0; c < 6; c++) m.e[c] = p[(size_t)c * st];
    }
    __device__ static void store(V *__restrict__ p, size_t st, const Mt<T> &m) {
#pragma unroll
        for (int c = 0; c < 9; c++) p[(size_t)c * st] = m.e[c];
    }
    static constexpr bool ROWS01_ONLY = false;
};

struct S32 {
    using T = float;
    using V = float4;
    static constexpr int NS = 3;
    static constexpr int BYTES = 48;
    __device__ static void load_rows01(const V *__restrict__ p, size_t st, Mt<T> &m) {
        float4 a = p[0], b = p[st], c = p[2 * st];
        m.e[0] = make_float2(a.x, a.y);
        m.e[1] = make_float2(a.z, a.w);
        m.e[2] = make_float2(b.x, b.y);
        m.e[3] = make_float2(b.z, b.w);
        m.e[4] = make_float2(c.x, c.y);
        m.e[5] = make_float2(c.z, c.w);
    }
    __device__ static void load(const V *__restrict__ p, size_t st, Mt<T> &m) {
        load_rows01(p, st, m);
        reconstruct_row2(m);
    }
    __device__ static void store(V *__restrict__ p, size_t st, const Mt<T> &m) {
        p[0] = make_float4(m.e[0].x, m.e[0].y, m.e[1].x, m.e[1].y);
        p[st] = make_float4(m.e[2].x, m.e[2].y, m.e[3].x, m.e[3].y);
        p[2 * st] = make_float4(m.e[4].x, m.e[4].y, m.e[5].x, m.e[5].y);
    }
    static constexpr bool ROWS01_ONLY = true;
};

template <class S>
__device__ __forceinline__ size_t su_idx(const Lat &l, int d, int par, uint32_t i) {
    return ((size_t)(d * l.npar + par) * S::NS) * l.vh + i;
}
template <class S>
__device__ __forceinline__ size_t sg_idx(const Lat &l, int par, uint32_t i) {
    return ((size_t)par * S::NS) * l.vh + i;
}

// ------------------------------------------------------------- the update --
// e2 density of a site from its w (see the header comment)
template <typename T>
__device__ __forceinline__ double e2_from_w(const Mt<T> &w) {
    double c1 = (double)w.e[1].y + (double)w.e[3].y;
    double c2 = (double)w.e[1].x - (double)w.e[3].x;
    double c3 = (double)w.e[0].y - (double)w.e[4].y;
    double c4 = (double)w.e[2].y + (double)w.e[6].y;
    double c5 = (double)w.e[2].x - (double)w.e[6].x;
    double c6 = (double)w.e[5].y + (double)w.e[7].y;
    double c7 = (double)w.e[5].x - (double)w.e[7].x;
    double c8 = ((double)w.e[0].y + (double)w.e[4].y - 2.0 * (double)w.e[8].y) * 0.57735026918962576451;
    return c1 * c1 + c2 * c2 + c3 * c3 + c4 * c4 + c5 * c5 + c6 * c6 + c7 * c7 + c8 * c8;
}

// one Cabibbo-Marinari hit on rows (A, B) of w, accumulated into g
template <int A, int B, typename T>
__device__ __forceinline__ void fsub_hit(Mt<T> &w, Mt<T> &g) {
    using C = typename CT<T>::t;
    T k0 = w.e[EL(A, A)].x + w.e[EL(B, B)].x;
    T k1 = -(w.e[EL(A, B)].y + w.e[EL(B, A)].y);
    T k2 = -(w.e[EL(A, B)].x - w.e[EL(B, A)].x);
    T k3 = -(w.e[EL(A, A)].y - w.e[EL(B, B)].y);
    T n = k0 * k0 + k1 * k1 + k2 * k2 + k3 * k3;
    if (n == T(0)) return;
    T r = frsqrt(n);
    k0 *= r;
    k1 *= r;
    k2 *= r;
    k3 *= r;
    const C x00 = mkc<C>(k0, k3), x01 = mkc<C>(k2, k1), x10 = mkc<C>(-k2, k1), x11 = mkc<C>(k0, -k3);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        C a = w.e[EL(A, c)], b = w.e[EL(B, c)];
        w.e[EL(A, c)] = fadd(fmul(x00, a), fmul(x01, b));
        w.e[EL(B, c)] = fadd(fmul(x10, a), fmul(x11, b));
        a = g.e[EL(A, c)];
        b = g.e[EL(B, c)];
        g.e[EL(A, c)] = fadd(fmul(x00, a), fmul(x01, b));
        g.e[EL(B, c)] = fadd(fmul(x10, a), fmul(x11, b));
    }
}

template <typename T>
__device__ __forceinline__ bool fproject(Mt<T> &m) {
    using C = typename CT<T>::t;
    T n0 = m.e[0].x * m.e[0].x + m.e[0].y * m.e[0].y + m.e[1].x * m.e[1].x + m.e[1].y * m.e[1].y +
           m.e[2].x * m.e[2].x + m.e[2].y * m.e[2].y;
    if (n0 == T(0)) return false;
    T r0 = frsqrt(n0);
#pragma unroll
    for (int k = 0; k < 3; k++) m.e[k] = mkc<C>(m.e[k].x * r0, m.e[k].y * r0);
    fcross_conj(&m.e[0], &m.e[3], &m.e[6]);
    T n2 = m.e[6].x * m.e[6].x + m.e[6].y * m.e[6].y + m.e[7].x * m.e[7].x + m.e[7].y * m.e[7].y +
           m.e[8].x * m.e[8].x + m.e[8].y * m.e[8].y;
    if (n2 == T(0)) return false;
    T r2 = frsqrt(n2);
#pragma unroll
    for (int k = 6; k < 9; k++) m.e[k] = mkc<C>(m.e[k].x * r2, m.e[k].y * r2);
    fcross_conj(&m.e[6], &m.e[0], &m.e[3]);
    return true;
}

template <typename T>
__device__ __forceinline__ void fidentity(Mt<T> &m) {
    using C = typename CT<T>::t;
#pragma unroll
    for (int k = 0; k < 9; k++) m.e[k] = mkc<C>((k % 4) == 0 ? T(1) : T(0), T(0));
}

// upd = Proj_SU3(I + omega (g - I)), g = w_final w^-1 accumulated by the hits
template <typename T>
__device__ __forceinline__ void fupdate(Mt<T> &w, T omega, unsigned hits, Mt<T> &g) {
    using C = typename CT<T>::t;
    fidentity(g);
#pragma unroll 1
    for (unsigned h = 0; h < hits; h++) {
        fsub_hit<0, 1>(w, g);
        fsub_hit<0, 2>(w, g);
        fsub_hit<1, 2>(w, g);
    }
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
            C x = g.e[EL(a, b)];
            g.e[EL(a, b)] = a == b ? mkc<C>(T(1) + omega * (x.x - T(1)), omega * x.y) : mkc<C>(omega * x.x, omega * x.y);
        }
    if (!fproject(g)) fidentity(g);
}

// c = a . b for the rows of c that storage S keeps
template <class S, typename T>
__device__ __forceinline__ void fprod_left(const Mt<T> &a, const Mt<T> &b, Mt<T> &c) {
    using C = typename CT<T>::t;
    constexpr int NR = S::ROWS01_ONLY ? 2 : 3;
#pragma unroll
    for (int i = 0; i < NR; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            C s = fmul(a.e[EL(i, 0)], b.e[EL(0, j)]);
            s = fadd(s, fmul(a.e[EL(i, 1)], b.e[EL(1, j)]));
            s = fadd(s, fmul(a.e[EL(i, 2)], b.e[EL(2, j)]));
            c.e[EL(i, j)] = s;
        }
}
// c = a . b^dagger (row-local in a: only the stored rows of a are needed)
template <class S, typename T>
__device__ __forceinline__ void fprod_dag(const Mt<T> &a, const Mt<T> &b, Mt<T> &c) {
    using C = typename CT<T>::t;
    constexpr int NR = S::ROWS01_ONLY ? 2 : 3;
#pragma unroll
    for (int i = 0; i < NR; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            C s = fmul_conj(a.e[EL(i, 0)], b.e[EL(j, 0)]);
            s = fadd(s, fmul_conj(a.e[EL(i, 1)], b.e[EL(j, 1)]));
            s = fadd(s, fmul_conj(a.e[EL(i, 2)], b.e[EL(j, 2)]));
            c.e[EL(i, j)] = s;
        }
}

// ----------------------------------------------------------- sweep kernel --
struct SweepArgs {
    Lat l;
    int par;
    double omega;
    unsigned hits;
    int track;          // 1: compute fused e2 partials
    double *part;       // [nt][nbx][2]
    unsigned *tickets;  // [nt + 1]
    double *slice;      // [nt][2] latest per-slice (pre, post) sums
    double *hist;       // [2 * hist_n]: (pre, post) totals per sweep index
    int sweep;          // this half-sweep's index
    int hist_n;
    unsigned *stop;     // stop word (0 = keep going); nullptr = never stop
    double tol_sum;     // stop when post(sweep-1) + pre(sweep) <= tol_sum
    unsigned *status;
};

constexpr int SWEEP_BLOCK = 128;

// deterministic sum of NQ values over the block; result in thread 0
template <int NQ>
__device__ __forceinline__ void fblock_sum(double (&v)[NQ], double (*sh)[SWEEP_BLOCK / 32]) {
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
            for (int k = 0; k < SWEEP_BLOCK / 32; k++) s += sh[q][k];
            v[q] = s;
        }
}

// Combine block partials: last block of a slice sums the slice, last slice sums
// all slices, applies the stopping test.  Called by all threads of the block.
__device__ void fused_reduce(const SweepArgs &a, double pre, double post) {
    __shared__ double sh[2][SWEEP_BLOCK / 32];
    __shared__ int last;
    double v[2] = {pre, post};
    fblock_sum<2>(v, sh);
    const uint32_t t = blockIdx.y, nbx = gridDim.x, nt = gridDim.y;
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
    // slice sum in index order
    if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0;
        const double *p = a.part + (size_t)t * nbx * 2;
        for (uint32_t b = 0; b < nbx; b++) {
            s0 += __ldcg(p + 2 * b);
            s1 += __ldcg(p + 2 * b + 1);
        }
        a.slice[2 * t] = s0;
        a.slice[2 * t + 1] = s1;
        a.tickets[t] = 0;
        __threadfence();
        unsigned tk = atomicAdd(&a.tickets[nt], 1u);
        last = tk == nt - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    double s0 = 0.0, s1 = 0.0;
    for (uint32_t q = 0; q < nt; q++) {
        s0 += __ldcg(a.slice + 2 * q);
        s1 += __ldcg(a.slice + 2 * q + 1);
    }
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
    if (a.stop && a.sweep >= 1 && a.sweep - 1 < a.hist_n) {
        double e2 = __ldcg(a.hist + 2 * (a.sweep - 1) + 1) + s0;
        if (e2 <= a.tol_sum) atomicExch(a.stop, (unsigned)(a.sweep + 1));
    }
}

template <class S>
__global__ void __launch_bounds__(SWEEP_BLOCK) k_sweep_fast(typename S::V *__restrict__ u,
                                                            typename S::V *__restrict__ g, SweepArgs a) {
    using T = typename S::T;
    using C = typename CT<T>::t;
    if (a.stop && *(volatile unsigned *)a.stop) return;
    const Lat &l = a.l;
    const uint32_t vsh = l.vs >> 1;
    const uint32_t off = blockIdx.x * SWEEP_BLOCK + threadIdx.x;
    const bool active = off < vsh;
    double pre = 0.0, post = 0.0;
    if (active) {
        const int par = a.par, op = par ^ 1;
        const uint32_t i = blockIdx.y * vsh + off;
        Coord c = coord_cb(l, par, i);
        uint32_t ib[3];
#pragma unroll
        for (int d = 0; d < 3; d++) ib[d] = back_L(l, c, d) >> 1;

        Mt<T> w;
#pragma unroll
        for (int k = 0; k < 9; k++) w.e[k] = mkc<C>(T(0), T(0));
#pragma unroll
        for (int d = 0; d < 3; d++) {
            Mt<T> f, r;
            S::load(u + su_idx<S>(l, d, par, i), l.vh, f);
            S::load(u + su_idx<S>(l, d, op, ib[d]), l.vh, r);
#pragma unroll
            for (int x = 0; x < 3; x++)
#pragma unroll
                for (int y = 0; y < 3; y++) w.e[EL(x, y)] = fadd(w.e[EL(x, y)], fadd(f.e[EL(x, y)], fconj(r.e[EL(y, x)])));
        }
        if (a.track) pre = e2_from_w(w);

        Mt<T> up;
        fupdate(w, (T)a.omega, a.hits, up);

        Mt<T> m, o;
        S::load(g + sg_idx<S>(l, par, i), l.vh, m);
        fprod_left<S>(up, m, o);
        S::store(g + sg_idx<S>(l, par, i), l.vh, o);
#pragma unroll
        for (int k = 0; k < 9; k++) w.e[k] = mkc<C>(T(0), T(0));
#pragma unroll
        for (int d = 0; d < 3; d++) {
            S::load(u + su_idx<S>(l, d, par, i), l.vh, m);
            fprod_left<S>(up, m, o);
            S::store(u + su_idx<S>(l, d, par, i), l.vh, o);
            if (a.track) {
                if (S::ROWS01_ONLY) reconstruct_row2(o);
#pragma unroll
                for (int k = 0; k < 9; k++) w.e[k] = fadd(w.e[k], o.e[k]);
            }
            // right multiplication is row-local: two-row storage needs no rebuild
            if (S::ROWS01_ONLY)
                S::load_rows01(u + su_idx<S>(l, d, op, ib[d]), l.vh, m);
            else
                S::load(u + su_idx<S>(l, d, op, ib[d]), l.vh, m);
            fprod_dag<S>(m, up, o);
            S::store(u + su_idx<S>(l, d, op, ib[d]), l.vh, o);
            if (a.track) {
                if (S::ROWS01_ONLY) reconstruct_row2(o);
#pragma unroll
                for (int x = 0; x < 3; x++)
#pragma unroll
                    for (int y = 0; y < 3; y++) w.e[EL(x, y)] = fadd(w.e[EL(x, y)], fconj(o.e[EL(y, x)]));
            }
        }
        if (a.track) post = e2_from_w(w);
    }
    if (a.track) fused_reduce(a, pre, post);
}

template <class S>
__global__ void k_reunit_fast(typename S::V *__restrict__ base, uint32_t stride, uint32_t nblk,
                              const unsigned *stop, unsigned *status) {
    if (stop && *(volatile const unsigned *)stop) return;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    if (i >= stride || k >= nblk) return;
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

__global__ void k_identity32(float4 *__restrict__ g, uint32_t stride, uint32_t nblk) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    if (i >= stride || k >= nblk) return;
    float4 *q = g + (size_t)k * 3 * stride + i;
    q[0] = make_float4(1.f, 0.f, 0.f, 0.f);
    q[stride] = make_float4(0.f, 0.f, 0.f, 0.f);
    q[2 * (size_t)stride] = make_float4(1.f, 0.f, 0.f, 0.f);
}

// ------------------------------------------------------------------ host --
static int ensure_track_buffers(gfc_ctx *c, int hist_n) {
    const Lat &l = c->lat;
    uint32_t nbx = ((l.vs >> 1) + SWEEP_BLOCK - 1) / SWEEP_BLOCK;
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
    uint32_t nbx = ((l.vs >> 1) + SWEEP_BLOCK - 1) / SWEEP_BLOCK;
    TrackPtrs t;
    t.part = c->part;
    t.slice = c->part + (size_t)l.nt * nbx * 2;
    t.tickets = c->tickets;
    t.stop = c->tickets + (l.nt + 1);
    return t;
}

template <class S>
static void launch_fast(gfc_ctx *c, typename S::V *u, typename S::V *g, int sweep, double omega, unsigned hits,
                        int track, unsigned *stop, double tol_sum) {
    const Lat &l = c->lat;
    TrackPtrs tp = track_ptrs(c);
    SweepArgs a;
    a.l = l;
    a.par = sweep & 1;
    a.omega = omega;
    a.hits = hits;
    a.track = track;
    a.part = tp.part;
    a.tickets = tp.tickets;
    a.slice = tp.slice;
    a.hist = c->e2_hist;
    a.sweep = sweep;
    a.hist_n = c->hist_n;
    a.stop = stop;
    a.tol_sum = tol_sum;
    a.status = c->dstatus;
    uint32_t nbx = ((l.vs >> 1) + SWEEP_BLOCK - 1) / SWEEP_BLOCK;
    k_sweep_fast<S><<<dim3(nbx, l.nt), SWEEP_BLOCK, 0, c->s>>>(u, g, a);
    c->launches++;
}

void launch_sweep_fast64(gfc_ctx *c, int sweep, double omega, unsigned hits, int track) {
    if (track && ensure_track_buffers(c, sweep + 1) != GFC_OK) return;
    if (!c->e2_hist) ensure_track_buffers(c, 1);
    launch_fast<S64>(c, c->u, c->g, sweep, omega, hits, track, nullptr, 0.0);
}

template <class S>
static void launch_reunit(gfc_ctx *c, typename S::V *base, uint32_t nblk, unsigned *stop) {
    const Lat &l = c->lat;
    dim3 grid((l.vh + 255) / 256, nblk);
    k_reunit_fast<S><<<grid, 256, 0, c->s>>>(base, l.vh, nblk, stop, c->dstatus);
    c->launches++;
}

static void print_res(int sweep, double res) { printf("Sweeps: %8d.\t residue: %3.2E \n", sweep, res); }

static int initial_proxy(gfc_ctx *c, const gfc_params *p, double *e2, double *res) {
    double th;
    int rc = gfc_ctx_e2(c, e2, &th);
    if (rc) return rc;
    *res = p->gfix_proxy == GFC_PROXY_THETA ? th : *e2;
    return GFC_OK;
}

// Run fused-e2 half-sweeps of storage S from sweep index `sweep` until the tracked
// e2 <= tol_e2 (stop word), `max_sweeps` is reached, or an error.  Returns the number
// of half-sweeps completed in *done (global index), and whether the stop fired.
template <class S>
static int run_until(gfc_ctx *c, typename S::V *u, typename S::V *g, int sweep0, int max_sweeps, double tol_e2,
                     double omega, unsigned hits, unsigned reunit, int *done, int *stopped) {
    const Lat &l = c->lat;
    int rc = ensure_track_buffers(c, max_sweeps + 2);
    if (rc) return rc;
    TrackPtrs tp = track_ptrs(c);
    GFC_CHECK(cudaMemsetAsync(tp.tickets, 0, (l.nt + 2) * sizeof(unsigned), c->s));
    const double tol_sum = tol_e2 * (double)l.v;
    const int chunk = 32;
    int sweep = sweep0;
    unsigned hstop = 0;
    *stopped = 0;
    while (sweep < max_sweeps) {
        int end = std::min(max_sweeps, sweep + chunk);
        for (; sweep < end; sweep++) {
            launch_fast<S>(c, u, g, sweep, omega, hits, 1, tp.stop, tol_sum);
            if (reunit && !((sweep + 1) % reunit)) {
                launch_reunit<S>(c, u, 3 * l.npar, tp.stop);
                launch_reunit<S>(c, g, l.npar, tp.stop);
            }
        }
        GFC_CHECK(cudaMemcpyAsync(c->hres + 16, tp.stop, sizeof(unsigned), cudaMemcpyDeviceToHost, c->s));
        GFC_CHECK(cudaStreamSynchronize(c->s));
        GFC_CHECK(cudaGetLastError());
        memcpy(&hstop, c->hres + 16, sizeof hstop);
        if (hstop) break;
    }
    if (hstop & 0x80000000u) {
        set_error("NaN in the gauge functional at half-sweep %u", hstop & 0x7fffffffu);
        return GFC_ERR_NUMERIC;
    }
    if (hstop) {
        *done = (int)hstop;
        *stopped = 1;
    } else {
        *done = sweep;
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
    int done = 0, stopped = 0;
    rc = run_until<S64>(c, c->u, c->g, 0, (int)p->max_sweeps_to_fix, tol_e2, (double)p->omega_OR, p->hits,
                        p->sweeps_to_reunitarization, &done, &stopped);
    if (rc) return rc;
    GFC_CHECK(cudaEventRecord(c->ev_d, c->s));
    r->sweeps = done;
    r->first_below_tol = stopped ? done - 1 : -1;
    r->site_updates = (long long)done * l.vh;
    return stopped ? done : GFC_FIX_NOT_CONVERGED;
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
    const size_t mat = (size_t)l.npar * l.vh * 9;
    // keep the FP64 links of the start; they are re-gauged at the switch
    GFC_CHECK(cudaMemcpyAsync(c->u0, c->u, 3 * mat * sizeof(double2), cudaMemcpyDeviceToDevice, c->s));
    {
        dim3 gu((l.vh + 255) / 256, 3 * l.npar), gg((l.vh + 255) / 256, l.npar);
        k_to_f32<<<gu, 256, 0, c->s>>>(c->u, (float4 *)c->u32, l.vh, 3 * l.npar);
        k_identity32<<<gg, 256, 0, c->s>>>((float4 *)c->g32, l.vh, l.npar);
        c->launches += 2;
    }
    // FP32 bulk
    const unsigned reunit32 = std::min<unsigned>(p->sweeps_to_reunitarization, 50u);
    int done = 0, stopped = 0;
    rc = run_until<S32>(c, (float4 *)c->u32, (float4 *)c->g32, 0, (int)p->max_sweeps_to_fix, sw,
                        (double)p->omega_OR, p->hits, reunit32, &done, &stopped);
    if (rc) return rc;
    r->sweeps_fp32 = done;
    if (!stopped) {
        r->sweeps = done;
        GFC_CHECK(cudaEventRecord(c->ev_d, c->s));
        return GFC_FIX_NOT_CONVERGED;
    }
    // switch: G in FP64 (rebuilt and projected), U = G U0 G^dagger from the FP64 start
    {
        dim3 gg((l.vh + 255) / 256, l.npar);
        k_to_f64<<<gg, 256, 0, c->s>>>((const float4 *)c->g32, c->g, l.vh, l.npar);
        c->launches++;
    }
    launch_apply_gt_spatial(c->u, c->u0, c->g, l, c->s);
    c->launches++;
    // FP64 refinement
    unsigned reunit64 = o->refine_reunit ? o->refine_reunit : p->sweeps_to_reunitarization;
    int done64 = 0;
    rc = run_until<S64>(c, c->u, c->g, done, (int)p->max_sweeps_to_fix, tol_e2, (double)p->omega_OR, p->hits,
                        reunit64, &done64, &stopped);
    if (rc) return rc;
    GFC_CHECK(cudaEventRecord(c->ev_d, c->s));
    r->sweeps = done64;
    r->first_below_tol = stopped ? done64 - 1 : -1;
    // site-updates in each precision
    r->site_updates = (long long)done64 * l.vh;
    return stopped ? done64 : GFC_FIX_NOT_CONVERGED;
}

}  // namespace gfc
