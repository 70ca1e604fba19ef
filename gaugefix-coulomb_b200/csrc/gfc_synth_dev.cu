// gfc_synth_dev.cu -- the seeded synthetic configuration built on the GPU.
//
// Same construction and random streams as host/gfc_synth.c:
//   U_mu(x) = g(x) exp(i s H_mu(x)) g(x+mu)^dagger, H = sum_a c_a lambda_a / 2,
//   c_a ~ N(0,1), g Haar on SU(3) (Gram-Schmidt of two Gaussian rows, third row
//   conj(r0 x r1)), exp by scaling and squaring of a degree-14 Taylor series.
// SplitMix64 streams keyed by (seed, site, slot) give bit-identical uniforms on host
// and device; the Box-Muller step uses the device log/sin/cos, whose last bits may
// differ from glibc's, so device-built links agree with host-built ones to rounding
// (~1e-16), not bit for bit.  Used where host generation of tens of GB would dominate
// (batches, serving requests); parity tests use the host generator.
#include <stdint.h>

#include "gfc_device.cuh"
#include "gfc_internal.h"

namespace gfc {

#define SYN_GOLDEN 0x9E3779B97F4A7C15ULL

__device__ __forceinline__ uint64_t syn_mix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

struct SynStream {
    uint64_t key, n;
    int have;
    double spare;
    __device__ SynStream(uint64_t seed, uint64_t site, unsigned slot) {
        key = syn_mix(syn_mix(seed + SYN_GOLDEN) + (site * 8u + slot + 1u) * 0xD1B54A32D192ED03ULL);
        n = 0;
        have = 0;
        spare = 0.0;
    }
    __device__ double uniform() {
        n++;
        uint64_t z = syn_mix(key + n * SYN_GOLDEN);
        return ((double)(z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    }
    __device__ double normal() {
        if (have) {
            have = 0;
            return spare;
        }
        double u1 = uniform(), u2 = uniform();
        double r = sqrt(-2.0 * log(u1));
        double s, c;
        sincos(6.283185307179586476925286766559 * u2, &s, &c);
        spare = r * s;
        have = 1;
        return r * c;
    }
};

__device__ void syn_mul(const M3 &a, const M3 &b, M3 &c) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            double re = 0, im = 0;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                re += a.e[EL(i, k)].x * b.e[EL(k, j)].x - a.e[EL(i, k)].y * b.e[EL(k, j)].y;
                im += a.e[EL(i, k)].x * b.e[EL(k, j)].y + a.e[EL(i, k)].y * b.e[EL(k, j)].x;
            }
            c.e[EL(i, j)] = make_double2(re, im);
        }
}

__device__ void syn_mul_dag(const M3 &a, const M3 &b, M3 &c) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            double re = 0, im = 0;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                re += a.e[EL(i, k)].x * b.e[EL(j, k)].x + a.e[EL(i, k)].y * b.e[EL(j, k)].y;
                im += a.e[EL(i, k)].y * b.e[EL(j, k)].x - a.e[EL(i, k)].x * b.e[EL(j, k)].y;
            }
            c.e[EL(i, j)] = make_double2(re, im);
        }
}

__device__ void syn_haar(SynStream &s, M3 &g) {
    double v[2][6];
    for (int r = 0; r < 2; r++)
        for (int k = 0; k < 6; k++) v[r][k] = s.normal();
    double n0 = 0;
    for (int k = 0; k < 6; k++) n0 += v[0][k] * v[0][k];
    n0 = 1.0 / sqrt(n0);
    for (int k = 0; k < 6; k++) v[0][k] *= n0;
    double pr = 0, pi = 0;
    for (int c = 0; c < 3; c++) {
        double ar = v[0][2 * c], ai = v[0][2 * c + 1], br = v[1][2 * c], bi = v[1][2 * c + 1];
        pr += ar * br + ai * bi;
        pi += ar * bi - ai * br;
    }
    for (int c = 0; c < 3; c++) {
        double ar = v[0][2 * c], ai = v[0][2 * c + 1];
        v[1][2 * c] -= pr * ar - pi * ai;
        v[1][2 * c + 1] -= pr * ai + pi * ar;
    }
    double n1 = 0;
    for (int k = 0; k < 6; k++) n1 += v[1][k] * v[1][k];
    n1 = 1.0 / sqrt(n1);
    for (int k = 0; k < 6; k++) v[1][k] *= n1;
    for (int c = 0; c < 3; c++) {
        g.e[EL(0, c)] = make_double2(v[0][2 * c], v[0][2 * c + 1]);
        g.e[EL(1, c)] = make_double2(v[1][2 * c], v[1][2 * c + 1]);
    }
    for (int c = 0; c < 3; c++) {
        int a = (c + 1) % 3, b = (c + 2) % 3;
        double2 r0a = g.e[EL(0, a)], r0b = g.e[EL(0, b)], r1a = g.e[EL(1, a)], r1b = g.e[EL(1, b)];
        double xr = r0a.x * r1b.x - r0a.y * r1b.y - (r0b.x * r1a.x - r0b.y * r1a.y);
        double xi = r0a.x * r1b.y + r0a.y * r1b.x - (r0b.x * r1a.y + r0b.y * r1a.x);
        g.e[EL(2, c)] = make_double2(xr, -xi);
    }
}

__device__ void syn_exp(SynStream &s, double scale, M3 &e) {
    double c[9];
    for (int a = 1; a <= 8; a++) c[a] = s.normal();
    const double r3 = 1.0 / sqrt(3.0);
    double hr[9] = {0}, hi[9] = {0};
    hr[0] = 0.5 * (c[3] + c[8] * r3);
    hr[4] = 0.5 * (-c[3] + c[8] * r3);
    hr[8] = 0.5 * (-2.0 * c[8] * r3);
    hr[1] = 0.5 * c[1]; hi[1] = -0.5 * c[2];
    hr[3] = 0.5 * c[1]; hi[3] = 0.5 * c[2];
    hr[2] = 0.5 * c[4]; hi[2] = -0.5 * c[5];
    hr[6] = 0.5 * c[4]; hi[6] = 0.5 * c[5];
    hr[5] = 0.5 * c[6]; hi[5] = -0.5 * c[7];
    hr[7] = 0.5 * c[6]; hi[7] = 0.5 * c[7];
    M3 x;
    double nrm = 0;
    for (int k = 0; k < 9; k++) {
        x.e[k] = make_double2(-scale * hi[k], scale * hr[k]);
        nrm += hr[k] * hr[k] + hi[k] * hi[k];
    }
    nrm = fabs(scale) * sqrt(nrm);
    int sq = 0;
    double f = 1.0;
    while (nrm * f > 0.25) {
        f *= 0.5;
        sq++;
    }
    for (int k = 0; k < 9; k++) x.e[k] = make_double2(x.e[k].x * f, x.e[k].y * f);
    M3 acc, tmp;
    set_identity(acc);
    for (int n = 14; n >= 1; n--) {
        syn_mul(x, acc, tmp);
        for (int k = 0; k < 9; k++) acc.e[k] = make_double2(tmp.e[k].x / (double)n, tmp.e[k].y / (double)n);
        for (int i = 0; i < 3; i++) acc.e[EL(i, i)].x += 1.0;
    }
    for (int k = 0; k < sq; k++) {
        syn_mul(acc, acc, tmp);
        acc = tmp;
    }
    e = acc;
}

// g(x) for every site into the (checkerboard SoA) field gtmp
__global__ void k_synth_g(Lat l, uint64_t seed, double2 *__restrict__ gtmp) {
    uint32_t L = blockIdx.x * blockDim.x + threadIdx.x;
    if (L >= l.v) return;
    SynStream st(seed, L, 4);
    M3 g;
    syn_haar(st, g);
    Slot s = slot_of(l, L);
    store_m(gtmp + gidx(l, s.par, 0, s.i), l.vh, g);
}

// U_mu(x) = g(x) exp(i s H) g(x+mu)^dagger for the 4 links of every site
__global__ void k_synth_links(Lat l, uint64_t seed, double scale, const double2 *__restrict__ gtmp,
                              double2 *__restrict__ u, double2 *__restrict__ ut) {
    uint32_t L = blockIdx.x * blockDim.x + threadIdx.x;
    if (L >= l.v) return;
    Coord c = coord_lex(l, L);
    Slot s = slot_of(l, L);
    M3 gx;
    load_m(gtmp + gidx(l, s.par, 0, s.i), l.vh, gx);
    for (int mu = 0; mu < 4; mu++) {
        uint32_t Ly = mu == 0 ? fwd_t_L(l, c) : fwd_L(l, c, mu - 1);
        Slot sy = slot_of(l, Ly);
        M3 gy, e, ge, uu;
        load_m(gtmp + gidx(l, sy.par, 0, sy.i), l.vh, gy);
        SynStream st(seed, L, (unsigned)mu);
        syn_exp(st, scale, e);
        syn_mul(gx, e, ge);
        syn_mul_dag(ge, gy, uu);
        double2 *dst = mu == 0 ? ut + gidx(l, s.par, 0, s.i) : u + uidx(l, mu - 1, s.par, 0, s.i);
        store_m(dst, l.vh, uu);
    }
}

void launch_synth(const Lat &l, uint64_t seed, double scale, double2 *gtmp, double2 *u, double2 *ut,
                  cudaStream_t s) {
    k_synth_g<<<(l.v + 127) / 128, 128, 0, s>>>(l, seed, gtmp);
    k_synth_links<<<(l.v + 127) / 128, 128, 0, s>>>(l, seed, scale, gtmp, u, ut);
}

}  // namespace gfc
