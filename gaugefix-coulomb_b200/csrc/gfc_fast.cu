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
    static constexpr bool ROWWISE = true;
    static constexpr int STORED_ROWS = 3;
};

// FP64, rows 0 and 1 only (6 double2 per matrix, 96 B); row 2 rebuilt as conj(r0 x r1)
struct S64R {
    using T = double;
    using V = double2;
    static constexpr int NS = 6;
    static constexpr int BYTES = 96;
    __device__ static void load_rows01(const V *__restrict__ p, size_t st, Mt<T> &m) {
#pragma unroll
        for (int c = 0; c < 6; c++) m.e[c] = p[(size_t)c * st];
    }
    __device__ static void load(const V *__restrict__ p, size_t st, Mt<T> &m) {
        load_rows01(p, st, m);
        reconstruct_row2(m);
    }
    __device__ static void store(V *__restrict__ p, size_t st, const Mt<T> &m) {
#pragma unroll
        for (int c = 0; c < 6; c++) p[(size_t)c * st] = m.e[c];
    }
    static constexpr bool ROWS01_ONLY = true;
    static constexpr bool ROWWISE = true;
    static constexpr int STORED_ROWS = 2;
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
    static constexpr bool ROWWISE = false;
    static constexpr int STORED_ROWS = 2;
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

// Contribution of row i = (o0, o1, o2) of a matrix o added to w (sign +1) or of
// o^dagger added to w (sign -1) to the 8 algebra components of w's e2 density:
//   c1 = Im w01 + Im w10, c2 = Re w01 - Re w10, c3 = Im w00 - Im w11,
//   c4 = Im w02 + Im w20, c5 = Re w02 - Re w20, c6 = Im w12 + Im w21,
//   c7 = Re w12 - Re w21, c8 = Im w00 + Im w11 - 2 Im w22 (times 1/sqrt 3 later).
// Adding o^dagger contributes exactly the negative of adding o.
template <int I, typename C>
__device__ __forceinline__ void acc_row(double (&c)[8], C o0, C o1, C o2, double s) {
    if (I == 0) {
        c[0] += s * o1.y;
        c[1] += s * o1.x;
        c[2] += s * o0.y;
        c[3] += s * o2.y;
        c[4] += s * o2.x;
        c[7] += s * o0.y;
    } else if (I == 1) {
        c[0] += s * o0.y;
        c[1] -= s * o0.x;
        c[2] -= s * o1.y;
        c[5] += s * o2.y;
        c[6] += s * o2.x;
        c[7] += s * o1.y;
    } else {
        c[3] += s * o0.y;
        c[4] -= s * o0.x;
        c[5] += s * o1.y;
        c[6] -= s * o1.x;
        c[7] -= 2.0 * s * o2.y;
    }
}

template <int I, typename T>
__device__ __forceinline__ void acc_mat_row(double (&c)[8], const Mt<T> &o, double s) {
    acc_row<I>(c, o.e[EL(I, 0)], o.e[EL(I, 1)], o.e[EL(I, 2)], s);
}

// f <- up . f for a forward link; FP64 works one row at a time to keep few values live
template <class S>
__device__ __forceinline__ void apply_forward(typename S::V *__restrict__ p, size_t st,
                                              const Mt<typename S::T> &up, int track, double (&cc)[8]) {
    using T = typename S::T;
    using C = typename CT<T>::t;
    Mt<T> f;
    S::load(p, st, f);
    if constexpr (S::ROWWISE) {
#pragma unroll
        for (int r = 0; r < 3; r++) {
            if (r >= S::STORED_ROWS && !track) break;   // row 2 of a two-row link: e2 only
            C o[3];
#pragma unroll
            for (int j = 0; j < 3; j++) {
                C s = fmul(up.e[EL(r, 0)], f.e[EL(0, j)]);
                s = fadd(s, fmul(up.e[EL(r, 1)], f.e[EL(1, j)]));
                s = fadd(s, fmul(up.e[EL(r, 2)], f.e[EL(2, j)]));
                o[j] = s;
                if (r < S::STORED_ROWS) p[(size_t)(3 * r + j) * st] = s;
            }
            if (track) {
                if (r == 0) acc_row<0>(cc, o[0], o[1], o[2], 1.0);
                if (r == 1) acc_row<1>(cc, o[0], o[1], o[2], 1.0);
                if (r == 2) acc_row<2>(cc, o[0], o[1], o[2], 1.0);
            }
        }
    } else {
        Mt<T> o;
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int j = 0; j < 3; j++) {
                C s = fmul(up.e[EL(r, 0)], f.e[EL(0, j)]);
                s = fadd(s, fmul(up.e[EL(r, 1)], f.e[EL(1, j)]));
                s = fadd(s, fmul(up.e[EL(r, 2)], f.e[EL(2, j)]));
                o.e[EL(r, j)] = s;
            }
        S::store(p, st, o);
        if (track) {
            acc_mat_row<0>(cc, o, 1.0);
            acc_mat_row<1>(cc, o, 1.0);
            acc_mat_row<2>(cc, o, 1.0);
        }
    }
}

// r <- r . up^dagger for a backward link (row-local)
template <class S>
__device__ __forceinline__ void apply_backward(typename S::V *__restrict__ p, size_t st,
                                               const Mt<typename S::T> &up, int track, double (&cc)[8]) {
    using T = typename S::T;
    using C = typename CT<T>::t;
    if constexpr (S::ROWWISE) {
        C rows[3][3];   // rows of the old link; row 2 of a two-row link is rebuilt for e2
#pragma unroll
        for (int r = 0; r < 3; r++) {
            if (r >= S::STORED_ROWS) {
                if (!track) break;
                fcross_conj(rows[0], rows[1], rows[2]);
            } else {
#pragma unroll
                for (int j = 0; j < 3; j++) rows[r][j] = p[(size_t)(3 * r + j) * st];
            }
            const C a0 = rows[r][0], a1 = rows[r][1], a2 = rows[r][2];
            C o[3];
#pragma unroll
            for (int j = 0; j < 3; j++) {
                C s = fmul_conj(a0, up.e[EL(j, 0)]);
                s = fadd(s, fmul_conj(a1, up.e[EL(j, 1)]));
                s = fadd(s, fmul_conj(a2, up.e[EL(j, 2)]));
                o[j] = s;
                if (r < S::STORED_ROWS) p[(size_t)(3 * r + j) * st] = s;
            }
            if (track) {
                if (r == 0) acc_row<0>(cc, o[0], o[1], o[2], -1.0);
                if (r == 1) acc_row<1>(cc, o[0], o[1], o[2], -1.0);
                if (r == 2) acc_row<2>(cc, o[0], o[1], o[2], -1.0);
            }
        }
    } else {
        Mt<T> m, o;
        if (track)
            S::load(p, st, m);
        else
            S::load_rows01(p, st, m);
        const int nr = track ? 3 : 2;
#pragma unroll
        for (int r = 0; r < 3; r++) {
            if (r >= nr) break;
#pragma unroll
            for (int j = 0; j < 3; j++) {
                C s = fmul_conj(m.e[EL(r, 0)], up.e[EL(j, 0)]);
                s = fadd(s, fmul_conj(m.e[EL(r, 1)], up.e[EL(j, 1)]));
                s = fadd(s, fmul_conj(m.e[EL(r, 2)], up.e[EL(j, 2)]));
                o.e[EL(r, j)] = s;
            }
        }
        S::store(p, st, o);
        if (track) {
            acc_mat_row<0>(cc, o, -1.0);
            acc_mat_row<1>(cc, o, -1.0);
            acc_mat_row<2>(cc, o, -1.0);
        }
    }
}

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
    unsigned *status;
};

// Launch shapes compiled into the library: (threads per block, minimum resident
// blocks per SM).  The second number caps registers per thread (65536 / (block *
// minb)); which shape is fastest depends on the lattice and is measured by
// gfc_ctx_autotune.
struct Shape {
    int block, minb;
};
constexpr Shape kShapes[] = {{128, 2}, {128, 3}, {128, 4}, {64, 4}, {64, 6}, {256, 1}, {256, 2}};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);
constexpr int MIN_BLOCK = 64;   // smallest block: sizes the per-block partial buffers

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
// all slices, applies the stopping test.  Called by all threads of the block.
template <int BLOCK>
__device__ void fused_reduce(const SweepArgs &a, double pre, double post) {
    __shared__ double sh[2][BLOCK / 32];
    __shared__ int last;
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
    // slice sum in index order
    if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0;
        const double *p = a.part + (size_t)t * nbx * 2;
        for (uint32_t b = 0; b < nbx; b++) {
            s0 += __ldcg(p + 2 * b);
            s1 += __ldcg(p + 2 * b + 1);
        }
        a.tickets[t] = 0;
        if (a.track == 2) {
            // slice-blocked sweeping: the whole-lattice test runs after the round
            double *r = a.ring + ((size_t)(a.sweep % a.ring_n) * a.l.nt + t) * 2;
            r[0] = s0;
            r[1] = s1;
            last = 0;
        } else {
            a.slice[2 * t] = s0;
            a.slice[2 * t + 1] = s1;
            __threadfence();
            unsigned tk = atomicAdd(&a.tickets[nt], 1u);
            last = tk == nt - 1;
        }
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

template <class S, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) k_sweep_fast(typename S::V *__restrict__ u,
                                                            typename S::V *__restrict__ g, SweepArgs a) {
    using T = typename S::T;
    using C = typename CT<T>::t;
    if (a.stop && *(volatile unsigned *)a.stop) return;
    const Lat &l = a.l;
    const uint32_t vsh = l.vs >> 1;
    const uint32_t off = blockIdx.x * BLOCK + threadIdx.x;
    const bool active = off < vsh;
    double pre = 0.0, post = 0.0;
    if (active) {
        const int par = a.par, op = par ^ 1;
        const uint32_t i = (a.t0 + blockIdx.y) * vsh + off;
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

        // G(x) <- up G(x)
        {
            Mt<T> m, o;
            S::load(g + sg_idx<S>(l, par, i), l.vh, m);
            fprod_left<S>(up, m, o);
            S::store(g + sg_idx<S>(l, par, i), l.vh, o);
        }
        // links; the post-update w(x) enters e2 only through its 8 algebra
        // components, accumulated row by row (see acc_row)
        double cc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int d = 0; d < 3; d++) {
            apply_forward<S>(u + su_idx<S>(l, d, par, i), l.vh, up, a.track, cc);
            apply_backward<S>(u + su_idx<S>(l, d, op, ib[d]), l.vh, up, a.track, cc);
        }
        if (a.track) {
            cc[7] *= 0.57735026918962576451;
#pragma unroll
            for (int k = 0; k < 8; k++) post += cc[k] * cc[k];
        }
    }
    if (a.track) fused_reduce<BLOCK>(a, pre, post);
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
    grid.x = ((a.l.vs >> 1) + B - 1) / B;
    k_sweep_fast<S, B, kShapes[K].minb><<<grid, B, 0, st>>>(u, g, a);
}

template <class S>
static void dispatch_fast(int v, dim3 grid, cudaStream_t st, typename S::V *u, typename S::V *g,
                          const SweepArgs &a) {
    switch (v) {
        case 0: launch_shape<S, 0>(grid, st, u, g, a); break;
        case 1: launch_shape<S, 1>(grid, st, u, g, a); break;
        case 2: launch_shape<S, 2>(grid, st, u, g, a); break;
        case 3: launch_shape<S, 3>(grid, st, u, g, a); break;
        case 4: launch_shape<S, 4>(grid, st, u, g, a); break;
        case 5: launch_shape<S, 5>(grid, st, u, g, a); break;
        default: launch_shape<S, 6>(grid, st, u, g, a); break;
    }
}

// One half-sweep of timeslices [t0, t0 + nsl) (all slices by default).
template <class S>
static void launch_fast(gfc_ctx *c, typename S::V *u, typename S::V *g, int sweep, double omega, unsigned hits,
                        int track, unsigned *stop, double tol_sum, int t0 = 0, int nsl = -1) {
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
    a.status = c->dstatus;
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

static void print_res(int sweep, double res) { printf("Sweeps: %8d.\t residue: %3.2E \n", sweep, res); }

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
                     double omega, unsigned hits, unsigned reunit, int *done, int *first_below) {
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
        const int chunk = 32;
        while (sweep < max_sweeps) {
            int end = std::min(max_sweeps, sweep + chunk);
            for (; sweep < end; sweep++) {
                launch_fast<S>(c, u, g, sweep, omega, hits, 1, tp.stop, tol_sum);
                if (reunit && !((sweep + 1) % reunit)) {
                    launch_reunit<S>(c, u, 3 * l.npar, tp.stop);
                    launch_reunit<S>(c, g, l.npar, tp.stop);
                }
            }
            if ((rc = read_stop(c, tp.stop, &hstop))) return rc;
            if (hstop) break;
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
                            p->sweeps_to_reunitarization, &done, &below);
        if (rc) return rc;
    } else {
        if ((rc = ensure_2row(c))) return rc;
        pack_2row(c);
        rc = run_until<S64R>(c, c->u64r, c->g64r, 0, (int)p->max_sweeps_to_fix, tol_e2, (double)p->omega_OR,
                             p->hits, p->sweeps_to_reunitarization, &done, &below);
        if (rc) return rc;
        unpack_2row(c);
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
    int done = 0, below = -1;
    rc = run_until<S32>(c, (float4 *)c->u32, (float4 *)c->g32, 0, (int)p->max_sweeps_to_fix, sw,
                        (double)p->omega_OR, p->hits, reunit32, &done, &below);
    if (rc) return rc;
    r->sweeps_fp32 = done;
    if (below < 0) {
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
    if ((rc = ensure_2row(c))) return rc;
    pack_2row(c);
    rc = run_until<S64R>(c, c->u64r, c->g64r, done, (int)p->max_sweeps_to_fix, tol_e2, (double)p->omega_OR,
                         p->hits, reunit64, &done64, &below);
    if (rc) return rc;
    unpack_2row(c);
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
//   [0..2] exact shapes, [3..9] FP64 fast shapes, [10..16] FP32 shapes (0: not timed).
using namespace gfc;

extern "C" int gfc_ctx_autotune(gfc_ctx *c, int which, double *times_out) {
    if (!c) return GFC_ERR_ARG;
    if (!c->has_links) return GFC_ERR_STATE;
    if (!which) which = 7;
    double times[GFC_TUNE_SLOTS] = {0.0};
    if (times_out)
        for (int k = 0; k < GFC_TUNE_SLOTS; k++) times_out[k] = 0.0;
    if (!c->lat.cb) return GFC_OK;   // odd ns: one serial kernel, nothing to choose
    GFC_CHECK(cudaSetDevice(c->dev));
    int rc = gfc_ctx_save_links(c);
    if (rc) return rc;
    const Lat &l = c->lat;
    const int n = 6;
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
        a.track = 1;
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
        for (int s = 0; s < exact_num_shapes(); s++) {
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
        for (int v = 0; v < kNumShapes; v++) {
            double t = timed(
                [&](int k) { dispatch_fast<S64R>(v, dim3(0, l.nt), c->s, c->u64r, c->g64r, args_for(k)); });
            times[3 + v] = t;
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
        for (int v = 0; v < kNumShapes; v++) {
            double t = timed([&](int k) {
                dispatch_fast<S32>(v, dim3(0, l.nt), c->s, (float4 *)c->u32, (float4 *)c->g32, args_for(k));
            });
            times[10 + v] = t;
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
        for (int v = 0; v < kNumShapes; v++)
            if (times[3 + v] > 0 && times[3 + v] < base) base = times[3 + v];
        rc = tune_blocking(S64R{}, c->u64r, c->g64r, 96, c->blk64_slices, c->blk64_sweeps, base, times + 17);
        if (rc) return rc;
    }
    if ((which & 4) && c->u32 && c->g32) {
        double base = 1e30;
        for (int v = 0; v < kNumShapes; v++)
            if (times[10 + v] > 0 && times[10 + v] < base) base = times[10 + v];
        rc = tune_blocking(S32{}, (float4 *)c->u32, (float4 *)c->g32, 48, c->blk32_slices, c->blk32_sweeps, base,
                           times + 21);
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
    if (exact >= exact_num_shapes() || fast64 >= kNumShapes || fast32 >= kNumShapes) return GFC_ERR_ARG;
    if (exact >= 0) c->shape_exact = exact;
    if (fast64 >= 0) c->shape_fast64 = fast64;
    if (fast32 >= 0) c->shape_fast32 = fast32;
    return GFC_OK;
}
