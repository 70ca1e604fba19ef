// gfc_fast_device.cuh -- device building blocks of the fast sweep kernels
// (storage policies, the direct-accumulation update, row-wise application with
// the fused e2 components).  Shared by the single-lattice kernels (gfc_fast.cu)
// and the batch engine (gfc_batch.cu).
#pragma once
#include <type_traits>

#include "gfc_device.cuh"
#include "gfc_internal.h"

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
    return mkc<C>(fma(a.x, b.x, -(a.y * b.y)), fma(a.x, b.y, a.y * b.x));
}
template <typename C>
__device__ __forceinline__ C fmul_conj(C a, C b) {  // a * conj(b)
    return mkc<C>(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -(a.x * b.y)));
}
template <typename C>
__device__ __forceinline__ C fadd(C a, C b) {
    return mkc<C>(a.x + b.x, a.y + b.y);
}
template <typename C>
__device__ __forceinline__ C fconj(C a) {
    return mkc<C>(a.x, -a.y);
}
// s + a b, s + a conj(b) and s - a b as chains of fused multiply-adds (four per
// complex product instead of two products, two fused operations and two sums).
// Every multiply-add of the fast update is written out as fma(): the compiler is
// left no choice of which products to fuse, so each launch shape of one kernel body
// computes the same bits.
template <typename C>
__device__ __forceinline__ C fmac(C s, C a, C b) {
    return mkc<C>(fma(-a.y, b.y, fma(a.x, b.x, s.x)), fma(a.y, b.x, fma(a.x, b.y, s.y)));
}
template <typename C>
__device__ __forceinline__ C fmac_conj(C s, C a, C b) {
    return mkc<C>(fma(a.y, b.y, fma(a.x, b.x, s.x)), fma(-a.x, b.y, fma(a.y, b.x, s.y)));
}
template <typename C>
__device__ __forceinline__ C fmsub(C s, C a, C b) {
    return mkc<C>(fma(a.y, b.y, fma(-a.x, b.x, s.x)), fma(-a.y, b.x, fma(-a.x, b.y, s.y)));
}

// FP32 complex arithmetic on paired single-precision instructions (one instruction
// does the same operation on both halves of a float2), two per complex multiply:
//   a b       = (a.x, a.x) * (b.x, b.y) + (-a.y, a.y) * (b.y, b.x)
//   a conj(b) = (a.x, a.y) * (b.x, b.x) + (a.y, -a.x) * (b.y, b.y)
// The real and imaginary parts are rounded like the fused scalar forms.
__device__ __forceinline__ float2 fadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 fmul(float2 a, float2 b) {
    return __ffma2_rn(make_float2(-a.y, a.y), make_float2(b.y, b.x), __fmul2_rn(make_float2(a.x, a.x), b));
}
__device__ __forceinline__ float2 fmac(float2 s, float2 a, float2 b) {
    s = __ffma2_rn(make_float2(a.x, a.x), b, s);
    return __ffma2_rn(make_float2(-a.y, a.y), make_float2(b.y, b.x), s);
}
__device__ __forceinline__ float2 fmul_conj(float2 a, float2 b) {
    return __ffma2_rn(make_float2(a.y, -a.x), make_float2(b.y, b.y), __fmul2_rn(a, make_float2(b.x, b.x)));
}
__device__ __forceinline__ float2 fmac_conj(float2 s, float2 a, float2 b) {
    s = __ffma2_rn(a, make_float2(b.x, b.x), s);
    return __ffma2_rn(make_float2(a.y, -a.x), make_float2(b.y, b.y), s);
}
__device__ __forceinline__ float2 fmsub(float2 s, float2 a, float2 b) {
    s = __ffma2_rn(make_float2(-a.x, -a.x), b, s);
    return __ffma2_rn(make_float2(a.y, -a.y), make_float2(b.y, b.x), s);
}

__device__ __forceinline__ double frsqrt(double x) { return rsqrt(x); }
__device__ __forceinline__ float frsqrt(float x) { return rsqrtf(x); }

// conj(a x b)
template <typename C>
__device__ __forceinline__ void fcross_conj(const C *a, const C *b, C *o) {
    o[0] = fconj(fmsub(fmul(a[1], b[2]), a[2], b[1]));
    o[1] = fconj(fmsub(fmul(a[2], b[0]), a[0], b[2]));
    o[2] = fconj(fmsub(fmul(a[0], b[1]), a[1], b[0]));
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
    double q = c1 * c1;
    q = fma(c2, c2, q);
    q = fma(c3, c3, q);
    q = fma(c4, c4, q);
    q = fma(c5, c5, q);
    q = fma(c6, c6, q);
    q = fma(c7, c7, q);
    return fma(c8, c8, q);
}

// e2 density of a site after its update: in a half-sweep the six links of x change
// only through x's own update, so w(x) afterwards is up . w(x) before it.  Used for
// FP64 storage, where it replaces the row-by-row accumulation from the six updated
// links (a third of the arithmetic); FP32 keeps the accumulation.
template <typename T>
__device__ __forceinline__ double e2_after(const Mt<T> &up, const Mt<T> &w0) {
    using C = typename CT<T>::t;
    Mt<T> wn;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
            C v = fmul(up.e[EL(a, 0)], w0.e[EL(0, b)]);
            v = fmac(v, up.e[EL(a, 1)], w0.e[EL(1, b)]);
            wn.e[EL(a, b)] = fmac(v, up.e[EL(a, 2)], w0.e[EL(2, b)]);
        }
    return e2_from_w(wn);
}

// Cabibbo-Marinari coefficients of the SU(2) subgroup on rows (A, B) of w: the
// embedded unit quaternion as x = {x_AA, x_AB, x_BA, x_BB}; false when the 2x2 block
// gives no direction (the hit is then the identity)
template <int A, int B, typename T>
__device__ __forceinline__ bool fsub_coef(const Mt<T> &w, typename CT<T>::t (&x)[4]) {
    using C = typename CT<T>::t;
    T k0 = w.e[EL(A, A)].x + w.e[EL(B, B)].x;
    T k1 = -(w.e[EL(A, B)].y + w.e[EL(B, A)].y);
    T k2 = -(w.e[EL(A, B)].x - w.e[EL(B, A)].x);
    T k3 = -(w.e[EL(A, A)].y - w.e[EL(B, B)].y);
    const T n = fma(k3, k3, fma(k2, k2, fma(k1, k1, k0 * k0)));
    if (n == T(0)) return false;
    T r = frsqrt(n);
    k0 *= r;
    k1 *= r;
    k2 *= r;
    k3 *= r;
    x[0] = mkc<C>(k0, k3);
    x[1] = mkc<C>(k2, k1);
    x[2] = mkc<C>(-k2, k1);
    x[3] = mkc<C>(k0, -k3);
    return true;
}
// rows (A, B) of m <- x . rows (A, B) of m
template <int A, int B, typename T>
__device__ __forceinline__ void frot_rows(Mt<T> &m, const typename CT<T>::t (&x)[4]) {
    using C = typename CT<T>::t;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const C a = m.e[EL(A, c)], b = m.e[EL(B, c)];
        m.e[EL(A, c)] = fmac(fmul(x[0], a), x[1], b);
        m.e[EL(B, c)] = fmac(fmul(x[2], a), x[3], b);
    }
}
// one Cabibbo-Marinari hit on rows (A, B) of w, accumulated into g
template <int A, int B, typename T>
__device__ __forceinline__ void fsub_hit(Mt<T> &w, Mt<T> &g) {
    typename CT<T>::t x[4];
    if (!fsub_coef<A, B>(w, x)) return;
    frot_rows<A, B>(w, x);
    frot_rows<A, B>(g, x);
}
// the first hit, starting from g = 1: the product of the three embedded subgroup
// elements is written out, without the products with the zeros and ones of the
// identity (which IEEE arithmetic does not let the compiler drop)
template <typename T>
__device__ __forceinline__ void fhit_first(Mt<T> &w, Mt<T> &g) {
    using C = typename CT<T>::t;
    C r[4], s[4], t[4];
    const C one = mkc<C>(T(1), T(0)), zero = mkc<C>(T(0), T(0));
    if (!fsub_coef<0, 1>(w, r)) r[0] = one, r[1] = zero, r[2] = zero, r[3] = one;
    frot_rows<0, 1>(w, r);
    if (!fsub_coef<0, 2>(w, s)) s[0] = one, s[1] = zero, s[2] = zero, s[3] = one;
    frot_rows<0, 2>(w, s);
    if (!fsub_coef<1, 2>(w, t)) t[0] = one, t[1] = zero, t[2] = zero, t[3] = one;
    frot_rows<1, 2>(w, t);
    // R = [[r0 r1 0] [r2 r3 0] [0 0 1]]; S acts on rows 0, 2; T on rows 1, 2
    const C g20 = fmul(s[2], r[0]), g21 = fmul(s[2], r[1]);
    g.e[0] = fmul(s[0], r[0]);
    g.e[1] = fmul(s[0], r[1]);
    g.e[2] = s[1];
    g.e[3] = fmac(fmul(t[0], r[2]), t[1], g20);
    g.e[4] = fmac(fmul(t[0], r[3]), t[1], g21);
    g.e[5] = fmul(t[1], s[3]);
    g.e[6] = fmac(fmul(t[2], r[2]), t[3], g20);
    g.e[7] = fmac(fmul(t[2], r[3]), t[3], g21);
    g.e[8] = fmul(t[3], s[3]);
}

// squared norm of a complex 3-vector as one chain of fused multiply-adds
template <typename C>
__device__ __forceinline__ decltype(C::x) fnorm2(C a, C b, C c) {
    decltype(C::x) n = a.x * a.x;
    n = fma(a.y, a.y, n);
    n = fma(b.x, b.x, n);
    n = fma(b.y, b.y, n);
    n = fma(c.x, c.x, n);
    return fma(c.y, c.y, n);
}

template <typename T>
__device__ __forceinline__ bool fproject(Mt<T> &m) {
    using C = typename CT<T>::t;
    const T n0 = fnorm2(m.e[0], m.e[1], m.e[2]);
    if (n0 == T(0)) return false;
    T r0 = frsqrt(n0);
#pragma unroll
    for (int k = 0; k < 3; k++) m.e[k] = mkc<C>(m.e[k].x * r0, m.e[k].y * r0);
    fcross_conj(&m.e[0], &m.e[3], &m.e[6]);
    const T n2 = fnorm2(m.e[6], m.e[7], m.e[8]);
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
    if (hits > 0)
        fhit_first(w, g);
    else
        fidentity(g);
#pragma unroll 1
    for (unsigned h = 1; h + 1 < hits; h++) {
        fsub_hit<0, 1>(w, g);
        fsub_hit<0, 2>(w, g);
        fsub_hit<1, 2>(w, g);
    }
    if (hits > 1) {   // the last hit written out: the entries of w that no later
                      // coefficient reads are not computed
        fsub_hit<0, 1>(w, g);
        fsub_hit<0, 2>(w, g);
        fsub_hit<1, 2>(w, g);
    }
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
            C x = g.e[EL(a, b)];
            g.e[EL(a, b)] = a == b ? mkc<C>(fma(omega, x.x - T(1), T(1)), omega * x.y)
                                   : mkc<C>(omega * x.x, omega * x.y);
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
            s = fmac(s, a.e[EL(i, 1)], b.e[EL(1, j)]);
            s = fmac(s, a.e[EL(i, 2)], b.e[EL(2, j)]);
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
            s = fmac_conj(s, a.e[EL(i, 1)], b.e[EL(j, 1)]);
            s = fmac_conj(s, a.e[EL(i, 2)], b.e[EL(j, 2)]);
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
                s = fmac(s, up.e[EL(r, 1)], f.e[EL(1, j)]);
                s = fmac(s, up.e[EL(r, 2)], f.e[EL(2, j)]);
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
                s = fmac(s, up.e[EL(r, 1)], f.e[EL(1, j)]);
                s = fmac(s, up.e[EL(r, 2)], f.e[EL(2, j)]);
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
                s = fmac_conj(s, a1, up.e[EL(j, 1)]);
                s = fmac_conj(s, a2, up.e[EL(j, 2)]);
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
                s = fmac_conj(s, m.e[EL(r, 1)], up.e[EL(j, 1)]);
                s = fmac_conj(s, m.e[EL(r, 2)], up.e[EL(j, 2)]);
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

// The e2 density of a site from its current links, without updating anything (the
// "pre" of fast_site on its own).  CB = false: the lexicographic layout of odd ns
// (one parity slot, i = the site's lexicographic index).
template <class S, bool CB = true>
__device__ __forceinline__ double measure_site(const typename S::V *__restrict__ u, const Lat &l, int par,
                                               uint32_t i) {
    using T = typename S::T;
    using C = typename CT<T>::t;
    if (!CB) par = 0;
    const int op = CB ? par ^ 1 : 0;
    Coord c = CB ? coord_cb(l, par, i) : coord_lex(l, i);
    Mt<T> w;
#pragma unroll
    for (int k = 0; k < 9; k++) w.e[k] = mkc<C>(T(0), T(0));
#pragma unroll
    for (int d = 0; d < 3; d++) {
        Mt<T> f, r;
        S::load(u + su_idx<S>(l, d, par, i), l.vh, f);
        S::load(u + su_idx<S>(l, d, op, CB ? back_L(l, c, d) >> 1 : back_L(l, c, d)), l.vh, r);
#pragma unroll
        for (int x = 0; x < 3; x++)
#pragma unroll
            for (int y = 0; y < 3; y++) w.e[EL(x, y)] = fadd(w.e[EL(x, y)], fadd(f.e[EL(x, y)], fconj(r.e[EL(y, x)])));
    }
    return e2_from_w(w);
}

// One site of a checkerboard half-sweep: w(x) from the three forward and three
// backward spatial links, the over-relaxed SU(3) update, G(x) <- up G(x) and the six
// links updated in place.  pre / post receive the site's contributions to e2 before
// and after the update (when track != 0).  u and g do not alias: with that known the
// compiler keeps the links it loaded for w(x) in registers for the link update
// instead of loading them again after the store to G.
template <class S>
__device__ __forceinline__ void fast_site(typename S::V *__restrict__ u, typename S::V *__restrict__ g,
                                          const Lat &l, int par, uint32_t i, typename S::T omega,
                                          unsigned hits, int track, double &pre, double &post) {
    using T = typename S::T;
    using C = typename CT<T>::t;
    const int op = par ^ 1;
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
    if (track) pre = e2_from_w(w);
    constexpr bool kPostW = std::is_same<T, double>::value;
    Mt<T> w0;
    if (kPostW && track) w0 = w;

    Mt<T> up;
    fupdate(w, omega, hits, up);
    const int track_links = kPostW ? 0 : track;

    // G(x) <- up G(x)
    {
        Mt<T> m, o;
        S::load(g + sg_idx<S>(l, par, i), l.vh, m);
        fprod_left<S>(up, m, o);
        S::store(g + sg_idx<S>(l, par, i), l.vh, o);
    }
    // links; the post-update w(x) enters e2 only through its 8 algebra components,
    // accumulated row by row (acc_row)
    double cc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int d = 0; d < 3; d++) {
        apply_forward<S>(u + su_idx<S>(l, d, par, i), l.vh, up, track_links, cc);
        apply_backward<S>(u + su_idx<S>(l, d, op, ib[d]), l.vh, up, track_links, cc);
    }
    if (track) {
        if constexpr (kPostW) {
            post = e2_after(up, w0);
        } else {
            cc[7] *= 0.57735026918962576451;
#pragma unroll
            for (int k = 0; k < 8; k++) post += cc[k] * cc[k];
        }
    }
}

// ------------------------------------------------- shared-memory staging --
// 16-byte asynchronous copy global -> shared (no registers held while in flight);
// both addresses 16-byte aligned.  wait_all makes the thread's own copies visible
// to that thread.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// up . f (forward link) or r . up^dagger (backward link) from a staged copy `src`
// (stride sst) to global `dst` (stride st); rows 0 and 1 are stored, row 2 only
// enters e2.  PROJ: the link is projected onto SU(3) before it is stored (a
// reunitarisation folded into the half-sweep).  projectSU3 reads rows 0 and 1 only,
// so the stored rows are those a separate pass would leave; a null row sets the
// status bit as that pass does.
template <class S, bool FWD, bool PROJ = false>
__device__ __forceinline__ void apply_staged(const typename S::V *src, int sst, typename S::V *__restrict__ dst,
                                             size_t st, const Mt<typename S::T> &up, int track, double (&cc)[8],
                                             unsigned *status = nullptr) {
    using T = typename S::T;
    using C = typename CT<T>::t;
    const double sg = FWD ? 1.0 : -1.0;
    if constexpr (S::ROWWISE && PROJ) {
        C r2[3];
        if (FWD || track) {
            C a[3] = {src[0], src[sst], src[2 * sst]};
            C b[3] = {src[3 * sst], src[4 * sst], src[5 * sst]};
            fcross_conj(a, b, r2);
        }
        Mt<T> o;
#pragma unroll
        for (int r = 0; r < 3; r++) {
            if (r == 2 && !track) break;
#pragma unroll
            for (int j = 0; j < 3; j++) {
                C v;
                if (FWD) {
                    v = fmul(up.e[EL(r, 0)], (C)src[j * sst]);
                    v = fmac(v, up.e[EL(r, 1)], (C)src[(3 + j) * sst]);
                    v = fmac(v, up.e[EL(r, 2)], r2[j]);
                } else {
                    const C m0 = r < 2 ? (C)src[(3 * r) * sst] : r2[0];
                    const C m1 = r < 2 ? (C)src[(3 * r + 1) * sst] : r2[1];
                    const C m2 = r < 2 ? (C)src[(3 * r + 2) * sst] : r2[2];
                    v = fmul_conj(m0, up.e[EL(j, 0)]);
                    v = fmac_conj(v, m1, up.e[EL(j, 1)]);
                    v = fmac_conj(v, m2, up.e[EL(j, 2)]);
                }
                o.e[EL(r, j)] = v;
            }
            if (track) {
                if (r == 0) acc_row<0>(cc, o.e[0], o.e[1], o.e[2], sg);
                if (r == 1) acc_row<1>(cc, o.e[3], o.e[4], o.e[5], sg);
                if (r == 2) acc_row<2>(cc, o.e[6], o.e[7], o.e[8], sg);
            }
        }
        if (!fproject(o) && status) atomicOr(status, GFC_STATUS_PROJECT_FAIL);
#pragma unroll
        for (int e = 0; e < 6; e++) dst[(size_t)e * st] = o.e[e];
    } else if constexpr (S::ROWWISE) {
        // one output row at a time; operands are read back from shared memory as
        // needed rather than held (row 2 of the link is rebuilt from rows 0 and 1)
        C r2[3];
        if (FWD || track) {
            C a[3] = {src[0], src[sst], src[2 * sst]};
            C b[3] = {src[3 * sst], src[4 * sst], src[5 * sst]};
            fcross_conj(a, b, r2);
        }
#pragma unroll
        for (int r = 0; r < 3; r++) {
            if (r == 2 && !track) break;
            C o[3];
#pragma unroll
            for (int j = 0; j < 3; j++) {
                C v;
                if (FWD) {
                    v = fmul(up.e[EL(r, 0)], (C)src[j * sst]);
                    v = fmac(v, up.e[EL(r, 1)], (C)src[(3 + j) * sst]);
                    v = fmac(v, up.e[EL(r, 2)], r2[j]);
                } else {
                    const C m0 = r < 2 ? (C)src[(3 * r) * sst] : r2[0];
                    const C m1 = r < 2 ? (C)src[(3 * r + 1) * sst] : r2[1];
                    const C m2 = r < 2 ? (C)src[(3 * r + 2) * sst] : r2[2];
                    v = fmul_conj(m0, up.e[EL(j, 0)]);
                    v = fmac_conj(v, m1, up.e[EL(j, 1)]);
                    v = fmac_conj(v, m2, up.e[EL(j, 2)]);
                }
                o[j] = v;
                if (r < 2) dst[(size_t)(3 * r + j) * st] = v;
            }
            if (track) {
                if (r == 0) acc_row<0>(cc, o[0], o[1], o[2], sg);
                if (r == 1) acc_row<1>(cc, o[0], o[1], o[2], sg);
                if (r == 2) acc_row<2>(cc, o[0], o[1], o[2], sg);
            }
        }
    } else {
        Mt<T> m, o;
        if (FWD || track)
            S::load(src, sst, m);
        else
            S::load_rows01(src, sst, m);   // rows 0 and 1 of r . up^dagger need rows 0 and 1 of r only
#pragma unroll
        for (int r = 0; r < 3; r++) {
            if (r == 2 && !track) break;
#pragma unroll
            for (int j = 0; j < 3; j++) {
                C v;
                if (FWD) {
                    v = fmul(up.e[EL(r, 0)], m.e[EL(0, j)]);
                    v = fmac(v, up.e[EL(r, 1)], m.e[EL(1, j)]);
                    v = fmac(v, up.e[EL(r, 2)], m.e[EL(2, j)]);
                } else {
                    v = fmul_conj(m.e[EL(r, 0)], up.e[EL(j, 0)]);
                    v = fmac_conj(v, m.e[EL(r, 1)], up.e[EL(j, 1)]);
                    v = fmac_conj(v, m.e[EL(r, 2)], up.e[EL(j, 2)]);
                }
                o.e[EL(r, j)] = v;
            }
        }
        if (track) {
            acc_mat_row<0>(cc, o, sg);
            acc_mat_row<1>(cc, o, sg);
            acc_mat_row<2>(cc, o, sg);
        }
        if constexpr (PROJ) {
            if (!fproject(o) && status) atomicOr(status, GFC_STATUS_PROJECT_FAIL);
        }
        S::store(dst, st, o);   // rows 0 and 1
    }
}

// fast_site with the links of the first NST / 2 directions (and, with SG, G) first
// copied into shared memory by cp.async: those bytes are requested at once, without
// registers held for them, and the link update reads them back from shared memory
// instead of from L2 (the links of the other directions are loaded from global
// memory twice, as in fast_site).  Staged layout per CTA: entry e of matrix m of
// thread x at sm[(m * NS + e) * BLOCK + x] (m = 2d forward, 2d+1 backward link of
// direction d, m = NST for G).  Two-row storage only.  CB = false: the lexicographic
// layout of odd ns (one parity slot, i = the site's lexicographic index).
// PROJ: the six links written are projected onto SU(3) first (apply_staged).
template <class S, int BLOCK, bool SG, int NST = 6, bool CB = true, bool PROJ = false>
__device__ __forceinline__ void fast_site_staged(typename S::V *__restrict__ u, typename S::V *__restrict__ g,
                                                 const Lat &l, int par, uint32_t i, typename S::T omega,
                                                 unsigned hits, int track, double &pre, double &post,
                                                 typename S::V *sm, unsigned *status = nullptr) {
    using T = typename S::T;
    using C = typename CT<T>::t;
    using V = typename S::V;
    static_assert(S::ROWS01_ONLY, "staging is for two-row storage");
    if (!CB) par = 0;
    const int op = CB ? par ^ 1 : 0;
    Coord c = CB ? coord_cb(l, par, i) : coord_lex(l, i);
    uint32_t ib[3];
#pragma unroll
    for (int d = 0; d < 3; d++) ib[d] = CB ? back_L(l, c, d) >> 1 : back_L(l, c, d);
    static_assert(NST == 2 || NST == 4 || NST == 6, "whole directions are staged");
    constexpr int ND = NST / 2;   // staged directions
    static_assert(!PROJ || ND == 3, "links are projected in the fully staged form only");
    V *my = sm + threadIdx.x;
#pragma unroll
    for (int d = 0; d < ND; d++) {
        const V *f = u + su_idx<S>(l, d, par, i);
        const V *r = u + su_idx<S>(l, d, op, ib[d]);
#pragma unroll
        for (int e = 0; e < S::NS; e++) {
            cp_async16(my + ((2 * d) * S::NS + e) * BLOCK, f + (size_t)e * l.vh);
            cp_async16(my + ((2 * d + 1) * S::NS + e) * BLOCK, r + (size_t)e * l.vh);
        }
    }
    if (SG) {
        const V *gp = g + sg_idx<S>(l, par, i);
#pragma unroll
        for (int e = 0; e < S::NS; e++) cp_async16(my + (NST * S::NS + e) * BLOCK, gp + (size_t)e * l.vh);
    }
    cp_async_wait_all();

    Mt<T> w;
#pragma unroll
    for (int k = 0; k < 9; k++) w.e[k] = mkc<C>(T(0), T(0));
#pragma unroll
    for (int d = 0; d < 3; d++) {
        Mt<T> f, r;
        if (d < ND) {
            S::load(my + (2 * d) * S::NS * BLOCK, BLOCK, f);
            S::load(my + (2 * d + 1) * S::NS * BLOCK, BLOCK, r);
        } else {
            S::load(u + su_idx<S>(l, d, par, i), l.vh, f);
            S::load(u + su_idx<S>(l, d, op, ib[d]), l.vh, r);
        }
#pragma unroll
        for (int x = 0; x < 3; x++)
#pragma unroll
            for (int y = 0; y < 3; y++) w.e[EL(x, y)] = fadd(w.e[EL(x, y)], fadd(f.e[EL(x, y)], fconj(r.e[EL(y, x)])));
    }
    if (track) pre = e2_from_w(w);
    constexpr bool kPostW = std::is_same<T, double>::value;
    Mt<T> w0;
    if (kPostW && track) w0 = w;

    Mt<T> up;
    fupdate(w, omega, hits, up);
    const int track_links = kPostW ? 0 : track;
    // the links are read again from shared memory below: keep the compiler from
    // holding the values loaded for w(x) in registers across the update instead
    asm volatile("" ::: "memory");
    {
        Mt<T> m, o;
        if (SG)
            S::load(my + NST * S::NS * BLOCK, BLOCK, m);
        else
            S::load(g + sg_idx<S>(l, par, i), l.vh, m);
        fprod_left<S>(up, m, o);
        S::store(g + sg_idx<S>(l, par, i), l.vh, o);
    }
    double cc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if constexpr (ND == 3) {
        // one copy of the direction body: the fully unrolled form outgrows the
        // instruction cache when many small blocks share an SM (3 % slower with
        // 32-site blocks); the operands come from shared memory, so the rolled loop
        // loses no load parallelism
#pragma unroll 1
        for (int d = 0; d < 3; d++) {
            const uint32_t b = d == 0 ? ib[0] : (d == 1 ? ib[1] : ib[2]);
            apply_staged<S, true, PROJ>(my + (2 * d) * S::NS * BLOCK, BLOCK, u + su_idx<S>(l, d, par, i), l.vh,
                                        up, track_links, cc, status);
            apply_staged<S, false, PROJ>(my + (2 * d + 1) * S::NS * BLOCK, BLOCK, u + su_idx<S>(l, d, op, b), l.vh,
                                         up, track_links, cc, status);
        }
    } else
#pragma unroll
    for (int d = 0; d < 3; d++) {
        if (d < ND) {
            apply_staged<S, true>(my + (2 * d) * S::NS * BLOCK, BLOCK, u + su_idx<S>(l, d, par, i), l.vh, up,
                                  track_links, cc);
            apply_staged<S, false>(my + (2 * d + 1) * S::NS * BLOCK, BLOCK, u + su_idx<S>(l, d, op, ib[d]), l.vh,
                                   up, track_links, cc);
        } else {
            apply_forward<S>(u + su_idx<S>(l, d, par, i), l.vh, up, track_links, cc);
            apply_backward<S>(u + su_idx<S>(l, d, op, ib[d]), l.vh, up, track_links, cc);
        }
    }
    if (track) {
        if constexpr (kPostW) {
            post = e2_after(up, w0);
        } else {
            cc[7] *= 0.57735026918962576451;
#pragma unroll
            for (int k = 0; k < 8; k++) post += cc[k] * cc[k];
        }
    }
}

}  // namespace gfc
