/*
 * Seeded synthetic SU(3) gauge configurations.
 *
 *   U_mu(x) = g(x) . exp(i s H_mu(x)) . g(x + mu)^dagger
 *   H_mu(x) = sum_{a=1..8} c_a lambda_a / 2,   c_a ~ N(0, 1)
 *   g(x)    Haar-random SU(3)
 *
 * The configuration is a random gauge transform of a smooth field, so its Coulomb
 * gauge is known to exist and the over-relaxation has a well-defined target.  The
 * layout produced is the SCIDAC order that the reference reads
 * (fields.h:39-43): [t][z][y][x][mu][row][col][re,im] with mu = 0 temporal and
 * mu = 1, 2, 3 the z, y, x directions (settings.h:57-60).
 *
 * Random numbers are counter based: every (seed, site, slot) owns an independent
 * SplitMix64 stream (Steele, Lea, Flood 2014), so the result does not depend on the
 * number of OpenMP threads.  Slots 0..3 feed H_mu, slot 4 feeds g.  Normal deviates
 * come from the Box-Muller transform.  The seed -> bits mapping is this project's
 * own; it is documented here and stays fixed so fixtures remain valid.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "gfc.h"

#define GOLDEN64 0x9E3779B97F4A7C15ULL

static inline uint64_t sm_mix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

typedef struct {
    uint64_t key;
    uint64_t n;
    int have_spare;
    double spare;
} stream_t;

static void stream_init(stream_t *s, uint64_t seed, uint64_t site, unsigned slot) {
    s->key = sm_mix(sm_mix(seed + GOLDEN64) + (site * 8u + slot + 1u) * 0xD1B54A32D192ED03ULL);
    s->n = 0;
    s->have_spare = 0;
    s->spare = 0.0;
}

/* uniform in the open interval (0, 1) */
static inline double stream_uniform(stream_t *s) {
    s->n++;
    uint64_t z = sm_mix(s->key + s->n * GOLDEN64);
    return ((double)(z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

static double stream_normal(stream_t *s) {
    if (s->have_spare) {
        s->have_spare = 0;
        return s->spare;
    }
    double u1 = stream_uniform(s), u2 = stream_uniform(s);
    double r = sqrt(-2.0 * log(u1));
    double th = 6.283185307179586476925286766559 * u2;
    s->spare = r * sin(th);
    s->have_spare = 1;
    return r * cos(th);
}

/* 3x3 complex matrices as 18 doubles, row major, (re, im) pairs */
typedef struct { double m[18]; } m33;

#define RE(A, i, j) ((A).m[2 * (3 * (i) + (j))])
#define IM(A, i, j) ((A).m[2 * (3 * (i) + (j)) + 1])

static void m33_mul(const m33 *a, const m33 *b, m33 *c) {
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double re = 0, im = 0;
            for (int k = 0; k < 3; k++) {
                re += RE(*a, i, k) * RE(*b, k, j) - IM(*a, i, k) * IM(*b, k, j);
                im += RE(*a, i, k) * IM(*b, k, j) + IM(*a, i, k) * RE(*b, k, j);
            }
            RE(*c, i, j) = re;
            IM(*c, i, j) = im;
        }
}

/* c = a . b^dagger */
static void m33_mul_dag(const m33 *a, const m33 *b, m33 *c) {
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double re = 0, im = 0;
            for (int k = 0; k < 3; k++) {
                re += RE(*a, i, k) * RE(*b, j, k) + IM(*a, i, k) * IM(*b, j, k);
                im += IM(*a, i, k) * RE(*b, j, k) - RE(*a, i, k) * IM(*b, j, k);
            }
            RE(*c, i, j) = re;
            IM(*c, i, j) = im;
        }
}

/* Haar SU(3): Gram-Schmidt on two complex Gaussian rows gives a uniformly
   distributed orthonormal 2-frame; the third row conj(r0 x r1) completes it to the
   unique SU(3) element with those rows. */
static void haar_su3(stream_t *s, m33 *g) {
    double v[2][6];
    for (int r = 0; r < 2; r++)
        for (int k = 0; k < 6; k++) v[r][k] = stream_normal(s);
    /* normalise row 0 */
    double n0 = 0;
    for (int k = 0; k < 6; k++) n0 += v[0][k] * v[0][k];
    n0 = 1.0 / sqrt(n0);
    for (int k = 0; k < 6; k++) v[0][k] *= n0;
    /* row1 -= <row0, row1> row0  (inner product conjugate-linear in row0) */
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
        RE(*g, 0, c) = v[0][2 * c];
        IM(*g, 0, c) = v[0][2 * c + 1];
        RE(*g, 1, c) = v[1][2 * c];
        IM(*g, 1, c) = v[1][2 * c + 1];
    }
    for (int c = 0; c < 3; c++) {
        int a = (c + 1) % 3, b = (c + 2) % 3;
        /* (r0 x r1)_c = r0_a r1_b - r0_b r1_a ; row2 = conj of it */
        double xr = RE(*g, 0, a) * RE(*g, 1, b) - IM(*g, 0, a) * IM(*g, 1, b)
                  - (RE(*g, 0, b) * RE(*g, 1, a) - IM(*g, 0, b) * IM(*g, 1, a));
        double xi = RE(*g, 0, a) * IM(*g, 1, b) + IM(*g, 0, a) * RE(*g, 1, b)
                  - (RE(*g, 0, b) * IM(*g, 1, a) + IM(*g, 0, b) * RE(*g, 1, a));
        RE(*g, 2, c) = xr;
        IM(*g, 2, c) = -xi;
    }
}

/* exp(i s H), H = sum_a c_a lambda_a / 2, by scaling and squaring of a Taylor series */
static void exp_su3(stream_t *s, double scale, m33 *e) {
    double c[9];
    for (int a = 1; a <= 8; a++) c[a] = stream_normal(s);
    const double r3 = 1.0 / sqrt(3.0);
    m33 h;
    memset(&h, 0, sizeof h);
    RE(h, 0, 0) = 0.5 * (c[3] + c[8] * r3);
    RE(h, 1, 1) = 0.5 * (-c[3] + c[8] * r3);
    RE(h, 2, 2) = 0.5 * (-2.0 * c[8] * r3);
    RE(h, 0, 1) = 0.5 * c[1]; IM(h, 0, 1) = -0.5 * c[2];
    RE(h, 1, 0) = 0.5 * c[1]; IM(h, 1, 0) = 0.5 * c[2];
    RE(h, 0, 2) = 0.5 * c[4]; IM(h, 0, 2) = -0.5 * c[5];
    RE(h, 2, 0) = 0.5 * c[4]; IM(h, 2, 0) = 0.5 * c[5];
    RE(h, 1, 2) = 0.5 * c[6]; IM(h, 1, 2) = -0.5 * c[7];
    RE(h, 2, 1) = 0.5 * c[6]; IM(h, 2, 1) = 0.5 * c[7];
    /* X = i s H */
    m33 x;
    double nrm = 0;
    for (int k = 0; k < 9; k++) {
        x.m[2 * k] = -scale * h.m[2 * k + 1];
        x.m[2 * k + 1] = scale * h.m[2 * k];
        nrm += h.m[2 * k] * h.m[2 * k] + h.m[2 * k + 1] * h.m[2 * k + 1];
    }
    nrm = fabs(scale) * sqrt(nrm);
    int sq = 0;
    double f = 1.0;
    while (nrm * f > 0.25) { f *= 0.5; sq++; }
    for (int k = 0; k < 18; k++) x.m[k] *= f;
    /* Taylor: E = I + X + X^2/2 + ... (Horner form, degree 14) */
    m33 acc, tmp;
    memset(&acc, 0, sizeof acc);
    for (int i = 0; i < 3; i++) RE(acc, i, i) = 1.0;
    for (int n = 14; n >= 1; n--) {
        m33_mul(&x, &acc, &tmp);
        for (int k = 0; k < 18; k++) acc.m[k] = tmp.m[k] / (double)n;
        for (int i = 0; i < 3; i++) RE(acc, i, i) += 1.0;
    }
    for (int k = 0; k < sq; k++) {
        m33_mul(&acc, &acc, &tmp);
        acc = tmp;
    }
    *e = acc;
}

/* Lexicographic site index of the reference: ((t*ns + z)*ns + y)*ns + x. */
static inline size_t site_index(int ns, int t, int z, int y, int x) {
    return (((size_t)t * ns + z) * ns + y) * ns + x;
}

int gfc_synth_config(int ns, int nt, uint64_t seed, double scale, double *U) {
    if (ns <= 0 || nt <= 0 || U == NULL) return GFC_ERR_ARG;
    const size_t V = (size_t)ns * ns * ns * nt;
    m33 *g = (m33 *)malloc(V * sizeof(m33));
    if (!g) return GFC_ERR_NOMEM;

    #pragma omp parallel for schedule(static)
    for (size_t L = 0; L < V; L++) {
        stream_t st;
        stream_init(&st, seed, L, 4);
        haar_su3(&st, &g[L]);
    }

    #pragma omp parallel for schedule(static)
    for (size_t L = 0; L < V; L++) {
        int x = (int)(L % ns), y = (int)((L / ns) % ns), z = (int)((L / ((size_t)ns * ns)) % ns);
        int t = (int)(L / ((size_t)ns * ns * ns));
        for (int mu = 0; mu < 4; mu++) {
            int xt = t, xz = z, xy = y, xx = x;
            switch (mu) {
                case 0: xt = (t + 1) % nt; break;
                case 1: xz = (z + 1) % ns; break;
                case 2: xy = (y + 1) % ns; break;
                default: xx = (x + 1) % ns; break;
            }
            stream_t st;
            stream_init(&st, seed, L, (unsigned)mu);
            m33 e, ge, u;
            exp_su3(&st, scale, &e);
            m33_mul(&g[L], &e, &ge);
            m33_mul_dag(&ge, &g[site_index(ns, xt, xz, xy, xx)], &u);
            memcpy(U + (L * 4 + mu) * 18, u.m, sizeof u.m);
        }
    }
    free(g);
    return GFC_OK;
}
