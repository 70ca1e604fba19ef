// gfc_device.cuh -- device-side lattice layout and SU(3) algebra.
//
// Two arithmetic flavours live here:
//   * "x" (exact) functions round exactly like the reference build
//     (gcc -std=c99, which turns FP contraction off): every product and sum is an
//     explicitly rounded __dmul_rn / __dadd_rn so the compiler can never fuse them,
//     complex products use the C99 expansion (ac - bd, ad + bc), complex quotients
//     use Smith's method, and |z| uses the hypot algorithm glibc ships.  Fused
//     multiply-adds appear only inside correctly rounded divisions (a method whose
//     result is the IEEE quotient), never in the reference's own arithmetic.  Kernels
//     built from these functions reproduce the reference's links and gauge
//     transformation bit for bit.
//   * "f" (fast) functions are templated on the storage precision and let the
//     compiler contract into FMA; they implement the same mathematics with fewer
//     operations (no explicit 3x3 inverse).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace gfc {

// ------------------------------------------------------------------ layout --
// Spatial links are stored structure-of-arrays and checkerboard ordered:
//   u[((d * 2 + par) * NC + c) * vh + i]      (d = 0,1,2 for z,y,x; c = matrix slot)
// with i the index of the site among the sites of parity par.  For even ns,
// i = L >> 1 where L = ((t*ns + z)*ns + y)*ns + x is the reference's site index
// (fields.h:33-43) and par = (x+y+z+t) & 1.  For odd ns the checkerboard cannot be
// split into independent halves, so the layout degenerates to one "parity" slot
// holding all V sites in lexicographic order (i = L, par = 0).
// Gauge transformation and temporal links use the same scheme without d.
struct Lat {
    int ns, nt;
    int cb;          // 1: checkerboard layout (even ns), 0: lexicographic (odd ns)
    uint32_t vs;     // spatial volume ns^3
    uint32_t v;      // volume
    uint32_t vh;     // sites per parity slot (v/2 or v)
    int npar;        // 2 or 1
};

__host__ __device__ inline Lat make_lat(int ns, int nt) {
    Lat l;
    l.ns = ns;
    l.nt = nt;
    l.cb = (ns % 2) == 0;
    l.vs = (uint32_t)ns * ns * ns;
    l.v = l.vs * (uint32_t)nt;
    l.npar = l.cb ? 2 : 1;
    l.vh = l.cb ? l.v / 2 : l.v;
    return l;
}

struct Slot {
    int par;
    uint32_t i;
};

__host__ __device__ __forceinline__ Slot slot_of(const Lat &l, uint32_t L) {
    Slot s;
    if (l.cb) {
        uint32_t x = L % l.ns, r = L / l.ns;
        uint32_t y = r % l.ns;
        r /= l.ns;
        uint32_t z = r % l.ns, t = r / l.ns;
        s.par = (int)((x + y + z + t) & 1u);
        s.i = L >> 1;
    } else {
        s.par = 0;
        s.i = L;
    }
    return s;
}

// coordinates of the site in slot (par, i) for the checkerboard layout
struct Coord {
    uint32_t x, y, z, t, L;
};

__host__ __device__ __forceinline__ Coord coord_cb(const Lat &l, int par, uint32_t i) {
    Coord c;
    uint32_t L0 = 2u * i;
    uint32_t x0 = L0 % l.ns, r = L0 / l.ns;
    c.y = r % l.ns;
    r /= l.ns;
    c.z = r % l.ns;
    c.t = r / l.ns;
    c.x = x0 + (((uint32_t)par ^ (c.y + c.z + c.t)) & 1u);
    c.L = L0 + (c.x - x0);
    return c;
}

__host__ __device__ __forceinline__ Coord coord_lex(const Lat &l, uint32_t L) {
    Coord c;
    c.L = L;
    c.x = L % l.ns;
    uint32_t r = L / l.ns;
    c.y = r % l.ns;
    r /= l.ns;
    c.z = r % l.ns;
    c.t = r / l.ns;
    return c;
}

// lexicographic index of the backward neighbour x - d (d = 0,1,2 for z,y,x)
__host__ __device__ __forceinline__ uint32_t back_L(const Lat &l, const Coord &c, int d) {
    uint32_t ns = l.ns;
    if (d == 0) return c.z ? c.L - ns * ns : c.L + (ns - 1) * ns * ns;
    if (d == 1) return c.y ? c.L - ns : c.L + (ns - 1) * ns;
    return c.x ? c.L - 1 : c.L + (ns - 1);
}
// The k-th site of parity p = (x + y + z + t) & 1 in lexicographic order, odd ns: row
// R (of ns sites along x) has row parity R & 1 (ns is odd, so R = y + ns z + ns^2 t has
// the parity of y + z + t), so the sites of parity p in a row are x = p ^ (R & 1), +2,
// ...; a pair of rows holds exactly ns of them, (ns + 1) / 2 in its first row when
// p = 0, (ns - 1) / 2 when p = 1.  False past the last one.
__device__ __forceinline__ bool odd_parity_site(const Lat &l, int p, uint32_t k, uint32_t &L) {
    const uint32_t ns = (uint32_t)l.ns;
    const uint32_t a = p ? (ns - 1) >> 1 : (ns + 1) >> 1;   // in the first (even) row of a pair
    const uint32_t pair = k / ns, rem = k - pair * ns;
    const uint32_t R = rem < a ? 2 * pair : 2 * pair + 1;
    const uint32_t j = rem < a ? rem : rem - a;
    const uint32_t x = 2 * j + ((uint32_t)p ^ (R & 1u));
    L = x + ns * R;
    return R < (uint32_t)l.ns * (uint32_t)l.ns * (uint32_t)l.nt;
}

__host__ __device__ __forceinline__ uint32_t fwd_L(const Lat &l, const Coord &c, int d) {
    uint32_t ns = l.ns;
    if (d == 0) return c.z + 1 < ns ? c.L + ns * ns : c.L - (ns - 1) * ns * ns;
    if (d == 1) return c.y + 1 < ns ? c.L + ns : c.L - (ns - 1) * ns;
    return c.x + 1 < ns ? c.L + 1 : c.L - (ns - 1);
}
__host__ __device__ __forceinline__ uint32_t fwd_t_L(const Lat &l, const Coord &c) {
    return c.t + 1 < (uint32_t)l.nt ? c.L + l.vs : c.L - (uint32_t)(l.nt - 1) * l.vs;
}

// element index of matrix slot c of link direction d
__host__ __device__ __forceinline__ size_t uidx(const Lat &l, int d, int par, int c, uint32_t i, int nc = 9) {
    return ((size_t)(d * l.npar + par) * nc + c) * l.vh + i;
}
__host__ __device__ __forceinline__ size_t gidx(const Lat &l, int par, int c, uint32_t i, int nc = 9) {
    return ((size_t)par * nc + c) * l.vh + i;
}

// ------------------------------------------------ exact complex arithmetic --
__device__ __forceinline__ double xm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xa(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xs(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xd(double a, double b) { return __ddiv_rn(a, b); }
// 1 / b correctly rounded: by IEEE round-to-nearest the same value as xd(1.0, b)
__device__ __forceinline__ double xrcp(double b) { return __drcp_rn(b); }

__device__ __forceinline__ double2 cz() { return make_double2(0.0, 0.0); }
__device__ __forceinline__ double2 xcadd(double2 a, double2 b) { return make_double2(xa(a.x, b.x), xa(a.y, b.y)); }
__device__ __forceinline__ double2 xcsub(double2 a, double2 b) { return make_double2(xs(a.x, b.x), xs(a.y, b.y)); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 xcmul(double2 a, double2 b) {
    return make_double2(xs(xm(a.x, b.x), xm(a.y, b.y)), xa(xm(a.x, b.y), xm(a.y, b.x)));
}

// |z| as glibc computes it: Borges, "An improved algorithm for hypot(a,b)" (2019),
// the correction step without fused multiply-add, with power-of-two rescaling for
// extreme exponents and the early exit for a negligible smaller operand.
// Both correction forms are evaluated and one is selected: the sites of a warp take
// either, so a branch would run both for the warp anyway.
__device__ __forceinline__ double xhypot_kernel(double ax, double ay) {
    const double h = __dsqrt_rn(xa(xm(ax, ax), xm(ay, ay)));
    const double da = xs(h, ay);
    const double t1a = xm(ax, xs(xm(2.0, da), ax));
    const double t2a = xm(xs(da, xm(2.0, xs(ax, ay))), da);
    const double db = xs(h, ax);
    const double t1b = xm(xm(2.0, db), xs(ax, xm(2.0, ay)));
    const double t2b = xa(xm(xs(xm(4.0, db), ay), ay), xm(db, db));
    const bool a = h <= xm(2.0, ay);
    return xs(h, xd(xa(a ? t1a : t1b, a ? t2a : t2b), xm(2.0, h)));
}
// extreme exponents, rescaled by powers of two (out of line: never met in a gauge field)
static __device__ __noinline__ double xhypot_scaled(double ax, double ay) {
    if (ax > 0x1p+500) return xm(xhypot_kernel(xm(ax, 0x1p-600), xm(ay, 0x1p-600)), 0x1p+600);
    return xm(xhypot_kernel(xm(ax, 0x1p+600), xm(ay, 0x1p+600)), 0x1p-600);
}
__device__ __forceinline__ double xhypot(double x, double y) {
    double ax = fabs(x), ay = fabs(y);
    if (ax < ay) {
        double t = ax;
        ax = ay;
        ay = t;
    }
    if (ay <= xm(ax, 0x1p-54)) return xa(ax, ay);
    if (ax > 0x1p+500 || ay < 0x1p-500) return xhypot_scaled(ax, ay);
    return xhypot_kernel(ax, ay);
}

// --------------------------------------------------------------- matrices --
struct M3 {
    double2 e[9];
};
#define EL(a, b) ((a) * 3 + (b))

__device__ __forceinline__ void set_identity(M3 &m) {
#pragma unroll
    for (int k = 0; k < 9; k++) m.e[k] = make_double2((k % 4) == 0 ? 1.0 : 0.0, 0.0);
}

// prod3x3 (SU3_ops.c:442-476): c_ab = ((0 + a_a0 b_0b) + a_a1 b_1b) + a_a2 b_2b
__device__ __forceinline__ void xprod(const M3 &a, const M3 &b, M3 &c) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            double2 s = cz();
#pragma unroll
            for (int k = 0; k < 3; k++) s = xcadd(s, xcmul(a.e[EL(i, k)], b.e[EL(k, j)]));
            c.e[EL(i, j)] = s;
        }
}
// a . b^dagger with the conjugate taken first (hermConj3x3 then prod3x3)
__device__ __forceinline__ void xprod_dag(const M3 &a, const M3 &b, M3 &c) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            double2 s = cz();
#pragma unroll
            for (int k = 0; k < 3; k++) s = xcadd(s, xcmul(a.e[EL(i, k)], cconj(b.e[EL(j, k)])));
            c.e[EL(i, j)] = s;
        }
}

// Smith division of every entry of num by the same complex d (inverse3x3's
// "/ a_det", SU3_ops.c:843-900); ratio and denominator do not depend on the entry.
// The two cases (|Re d| < |Im d| or not) differ only in which operands enter the
// same sequence of rounded operations, so the operands are selected instead of
// branched on: sites of one warp take different cases, and a branch would run the
// divisions of both for the whole warp.  The results are those of the branches.
//
// All eighteen quotients share the denominator, so they are formed from its
// correctly rounded reciprocal y by Markstein's method (P. Markstein, "Computation
// of elementary functions on the IBM RISC System/6000 processor", IBM J. Res. Dev.
// 34 (1990)): q0 = RN(a y) is within two ulps of a/b; with the remainder
// r = a - b q, exact by fused multiply-add once q is within one ulp, q1 = RN(q0 + r0 y)
// is within one ulp and q2 = RN(q1 + r1 y) is the correctly rounded a/b, the value
// of IEEE division.  The argument needs the operands, quotient and remainder clear
// of underflow and overflow; outside [2^-500, 2^500] the division is done directly.
// A zero dividend gives q0, a zero of the quotient's sign.
__device__ __forceinline__ bool xdiv_in_range(double a) {
    const double x = fabs(a);
    return x >= 0x1p-500 && x <= 0x1p+500;
}
__device__ __forceinline__ double xdiv_by_rcp(double a, double b, double y) {
    const double q0 = __dmul_rn(a, y);
    const double r0 = __fma_rn(-b, q0, a);
    const double q1 = __fma_rn(r0, y, q0);
    const double r1 = __fma_rn(-b, q1, a);
    const double q2 = __fma_rn(r1, y, q1);
    return a == 0.0 ? q0 : q2;
}
// The plain division out of line: operands outside the range never occur in a
// gauge field, and one shared copy keeps the kernels' code (and instruction-cache
// misses) smaller than eighteen inlined ones.
static __device__ __noinline__ double xd_rare(double a, double b) { return __ddiv_rn(a, b); }
// a / b for a divisor b shared by several quotients: y = xrcp(b), b_ok =
// xdiv_in_range(b); equal to xd(a, b) for every a and b
__device__ __forceinline__ double xdiv_shared(double a, double b, double y, bool b_ok) {
    if (b_ok && (a == 0.0 || xdiv_in_range(a))) return xdiv_by_rcp(a, b, y);
    return xd_rare(a, b);
}

struct SmithDen {
    double r, den, rcp;
    int c_ge_d, tiny, rcp_ok;
};
__device__ __forceinline__ SmithDen smith_prepare(double2 dd) {
    SmithDen s;
    const double c = dd.x, d = dd.y;
    s.c_ge_d = !(fabs(c) < fabs(d));
    const double num = s.c_ge_d ? d : c, dnm = s.c_ge_d ? c : d;   // r = d/c or c/d
    s.r = xd(num, dnm);
    s.den = xa(xm(num, s.r), dnm);                                   // d r + c or c r + d
    s.tiny = !(fabs(s.r) > 2.2250738585072014e-308);
    s.rcp = xrcp(s.den);
    s.rcp_ok = xdiv_in_range(s.den);
    return s;
}
// Smith's form for a ratio below the smallest normal number (never met in a gauge
// field; out of line to keep the kernels' code small)
static __device__ __noinline__ double2 smith_div_tiny(double a, double b, double c, double d, double den, int c_ge_d) {
    if (!c_ge_d) return make_double2(xd(xa(xm(c, xd(a, d)), b), den), xd(xs(xm(c, xd(b, d)), a), den));
    return make_double2(xd(xa(a, xm(d, xd(b, c))), den), xd(xs(b, xm(d, xd(a, c))), den));
}
__device__ __forceinline__ double2 smith_div(double2 x, double2 dd, const SmithDen &s) {
    const double a = x.x, b = x.y, c = dd.x, d = dd.y;
    if (!s.tiny) {
        // c >= d: re = (b r + a) / den, im = (b - a r) / den
        // c <  d: re = (a r + b) / den, im = (b r - a) / den
        const double p = s.c_ge_d ? b : a, q = s.c_ge_d ? a : b;
        const double t = xm(q, s.r);
        const double hi = s.c_ge_d ? b : t, lo = s.c_ge_d ? t : a;
        return make_double2(xdiv_shared(xa(xm(p, s.r), q), s.den, s.rcp, s.rcp_ok),
                            xdiv_shared(xs(hi, lo), s.den, s.rcp, s.rcp_ok));
    }
    return smith_div_tiny(a, b, c, d, s.den, s.c_ge_d);
}

// determinant3x3 (SU3_ops.c:251-281)
__device__ __forceinline__ double2 xdet(const M3 &m) {
    const double2 *e = m.e;
    double2 t0 = xcmul(e[EL(0, 0)], xcsub(xcmul(e[EL(1, 1)], e[EL(2, 2)]), xcmul(e[EL(1, 2)], e[EL(2, 1)])));
    double2 t1 = xcmul(e[EL(0, 1)], xcsub(xcmul(e[EL(1, 2)], e[EL(2, 0)]), xcmul(e[EL(1, 0)], e[EL(2, 2)])));
    double2 t2 = xcmul(e[EL(0, 2)], xcsub(xcmul(e[EL(1, 0)], e[EL(2, 1)]), xcmul(e[EL(1, 1)], e[EL(2, 0)])));
    return xcadd(xcadd(t0, t1), t2);
}

// inverse3x3 (SU3_ops.c:843-900); returns Re(det) like the reference
__device__ __forceinline__ double xinverse(const M3 &a, M3 &ai) {
    const double2 *m = a.e;
    double2 d = xdet(a);
    if (d.x != 0.0 || d.y != 0.0) {
        SmithDen s = smith_prepare(d);
#define XCOF(p, q, r, t) xcsub(xcmul(m[p], m[q]), xcmul(m[r], m[t]))
        ai.e[EL(0, 0)] = smith_div(XCOF(EL(1, 1), EL(2, 2), EL(1, 2), EL(2, 1)), d, s);
        ai.e[EL(0, 1)] = smith_div(XCOF(EL(0, 2), EL(2, 1), EL(0, 1), EL(2, 2)), d, s);
        ai.e[EL(0, 2)] = smith_div(XCOF(EL(0, 1), EL(1, 2), EL(0, 2), EL(1, 1)), d, s);
        ai.e[EL(1, 0)] = smith_div(XCOF(EL(1, 2), EL(2, 0), EL(1, 0), EL(2, 2)), d, s);
        ai.e[EL(1, 1)] = smith_div(XCOF(EL(0, 0), EL(2, 2), EL(0, 2), EL(2, 0)), d, s);
        ai.e[EL(1, 2)] = smith_div(XCOF(EL(0, 2), EL(1, 0), EL(0, 0), EL(1, 2)), d, s);
        ai.e[EL(2, 0)] = smith_div(XCOF(EL(1, 0), EL(2, 1), EL(1, 1), EL(2, 0)), d, s);
        ai.e[EL(2, 1)] = smith_div(XCOF(EL(0, 1), EL(2, 0), EL(0, 0), EL(2, 1)), d, s);
        ai.e[EL(2, 2)] = smith_div(XCOF(EL(0, 0), EL(1, 1), EL(0, 1), EL(1, 0)), d, s);
#undef XCOF
    } else {
#pragma unroll
        for (int k = 0; k < 9; k++) ai.e[k] = cz();
    }
    return d.x;
}

// normalize3Vec (SU3_ops.c:903-951): r = sum |v_a|^2 with |.| = cabs
__device__ __forceinline__ int xnormalize(double2 v[3]) {
    double r = 0.0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        double h = xhypot(v[a].x, v[a].y);
        r = xa(r, xm(h, h));
    }
    if (r != 0.0) {
        r = xrcp(__dsqrt_rn(r));
#pragma unroll
        for (int a = 0; a < 3; a++) v[a] = make_double2(xm(v[a].x, r), xm(v[a].y, r));
        return 0;
    }
    return -1;
}

// crossproductConj (SU3_ops.c:954-989)
__device__ __forceinline__ void xcross_conj(const double2 u[3], const double2 v[3], double2 w[3]) {
    w[0] = cconj(xcsub(xcmul(u[1], v[2]), xcmul(u[2], v[1])));
    w[1] = cconj(xcsub(xcmul(u[2], v[0]), xcmul(u[0], v[2])));
    w[2] = cconj(xcsub(xcmul(u[0], v[1]), xcmul(u[1], v[0])));
}

// projectSU3 (SU3_ops.c:994-1049); returns 0 on success, -1 on a null row
__device__ __forceinline__ int xproject(M3 &x) {
    double2 v0[3], v1[3], v2[3];
#pragma unroll
    for (int b = 0; b < 3; b++) {
        v0[b] = x.e[EL(0, b)];
        v1[b] = x.e[EL(1, b)];
    }
    int st = xnormalize(v0);
    xcross_conj(v0, v1, v2);
    st |= xnormalize(v2);
    xcross_conj(v2, v0, v1);
#pragma unroll
    for (int b = 0; b < 3; b++) {
        x.e[EL(0, b)] = v0[b];
        x.e[EL(1, b)] = v1[b];
        x.e[EL(2, b)] = v2[b];
    }
    return st ? -1 : 0;
}

// updateSubLosAlamos (SU3_ops.c:776-840), projectSU2 (SU2_ops.c:369-402),
// accumProdSU2_3x3 (SU3_ops.c:636-685); sub R = (0,1), S = (0,2), T = (1,2)
template <int A, int B>
__device__ __forceinline__ void xsub_los_alamos(M3 &w) {
    double2 *m = w.e;
    double k0 = xa(m[EL(A, A)].x, m[EL(B, B)].x);
    double k1 = -xa(m[EL(A, B)].y, m[EL(B, A)].y);
    double k2 = -xs(m[EL(A, B)].x, m[EL(B, A)].x);
    double k3 = -xs(m[EL(A, A)].y, m[EL(B, B)].y);
    double det = xa(xa(xa(xa(0.0, xm(k0, k0)), xm(k1, k1)), xm(k2, k2)), xm(k3, k3));
    if (det == 0.0) return;
    double inv = xrcp(__dsqrt_rn(det));
    k0 = xm(inv, k0);
    k1 = xm(inv, k1);
    k2 = xm(inv, k2);
    k3 = xm(inv, k3);
    double2 x00 = make_double2(k0, k3), x01 = make_double2(k2, k1);
    double2 x10 = make_double2(-k2, k1), x11 = make_double2(k0, -k3);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        double2 ga = m[EL(A, c)], gb = m[EL(B, c)];
        m[EL(A, c)] = xcadd(xcmul(x00, ga), xcmul(x01, gb));
        m[EL(B, c)] = xcadd(xcmul(x10, ga), xcmul(x11, gb));
    }
}

// gaugefixOverrelaxationLocal's update (gauge_fixing.c:537-596, 684-705):
// Los Alamos hits on w via the explicit inverse, then the omega binomial and the
// SU(3) projection (identity if the projection fails).
__device__ __forceinline__ void xor_update(M3 &w, double omega, unsigned hits, M3 &upd) {
    M3 winv, la;
    if (xinverse(w, winv) != 0.0) {
        for (unsigned h = 1; h <= hits; h++) {
            xsub_los_alamos<0, 1>(w);
            xsub_los_alamos<0, 2>(w);
            xsub_los_alamos<1, 2>(w);
        }
    }
    xprod(w, winv, la);
    // power3x3Binomial (SU3_ops.c:734-771)
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
            double2 x = la.e[EL(a, b)];
            upd.e[EL(a, b)] = a == b ? make_double2(xa(1.0, xm(omega, xs(x.x, 1.0))), xm(omega, x.y))
                                     : make_double2(xm(omega, x.x), xm(omega, x.y));
        }
    if (xproject(upd)) set_identity(upd);
}

// ------------------------------------------------------------- SoA access --
template <int NC = 9>
__device__ __forceinline__ void load_m(const double2 *__restrict__ base, size_t stride, M3 &m) {
#pragma unroll
    for (int c = 0; c < 9; c++) m.e[c] = base[(size_t)c * stride];
}
__device__ __forceinline__ void store_m(double2 *__restrict__ base, size_t stride, const M3 &m) {
#pragma unroll
    for (int c = 0; c < 9; c++) base[(size_t)c * stride] = m.e[c];
}

}  // namespace gfc
