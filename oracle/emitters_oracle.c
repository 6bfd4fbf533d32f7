/*
 * ORACLE -- test infrastructure only.
 *
 * CPU restatement of the device emitter sources (the reference's simulation
 * objects, idi/simulation/simobj.py) with the streams the device draws from:
 * emitter j of image b uses counter (0, j, (first + b) | 2^61, stream); the
 * per-image rotation counter (0, 2^64 - 1, (first + b) | 2^61, stream); the
 * key of site i in round r counter (1, i, (first + b) | 2^60 | r << 44, stream)
 * (one block, word 0).
 *
 *  - sphere: rndSphere (idi/util/random.py:39-51)
 *  - gnorm: normal (rho = 2) or generalised normal through Gamma(1/rho)
 *    (idi/util/random.py:6-26), Gamma by Marsaglia and Tsang (2000)
 *  - foil: simobj.py:738-760 with rndtruncexp (idi/util/random.py:142-151)
 *  - sites: crystal.updatePos (simobj.py:446-487) as weighted sampling without
 *    replacement by exponential keys (Efraimidis and Spirakis 2006): the k
 *    smallest keys by (key, site index), written in site order.
 */
#define _DEFAULT_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "philox_oracle.h"

#define EMIT_TAG (1ull << 61)
#define SITE_TAG (1ull << 60)

static double normal(stream_t *st) {
    const double a = stream_uniform(st);
    const double b = stream_uniform(st);
    return box_muller(a, b);
}

static double gamma_draw(double a, stream_t *st) {
    double boost = 1.0;
    if (a < 1.0) {
        boost = pow(1.0 - stream_uniform(st), 1.0 / a);
        a += 1.0;
    }
    const double d = a - 1.0 / 3.0, c = 1.0 / sqrt(9.0 * d);
    for (int trial = 0; trial < 1000; ++trial) {
        double x, v;
        int inner = 0;
        do {
            x = normal(st);
            v = 1.0 + c * x;
        } while (v <= 0.0 && ++inner < 1000);
        v = v * v * v;
        const double u = 1.0 - stream_uniform(st);
        const double x2 = x * x;
        if (u < 1.0 - 0.0331 * x2 * x2) return d * v * boost;
        if (log(u) < 0.5 * x2 + d * (1.0 - v + log(v))) return d * v * boost;
    }
    return -1.0;
}

static double gennorm(double fwhm, double rho, stream_t *st) {
    const double sign = stream_uniform(st) < 0.5 ? -1.0 : 1.0;
    const double g = gamma_draw(1.0 / rho, st);
    return fwhm * 0.5 * pow(fmax(g, 0.0) / log(2.0), 1.0 / rho) * sign;
}

static void rot3(const double *M, const double *v, double *o) {
    o[0] = M[0] * v[0] + M[1] * v[1] + M[2] * v[2];
    o[1] = M[3] * v[0] + M[4] * v[1] + M[5] * v[2];
    o[2] = M[6] * v[0] + M[7] * v[1] + M[8] * v[2];
}

/* kind: 0 sphere, 1 gnorm, 2 foil; out (n_images * n, 4) */
void orc_emit(int kind, int32_t n_images, int64_t n, double r, const double fwhm[3], const double rho[3], double depth,
              double attenuation, const double rot[9], int random_phase, uint64_t k0, uint64_t k1, uint64_t stream,
              uint64_t first, double *out) {
    for (int32_t b = 0; b < n_images; ++b) {
        for (int64_t j = 0; j < n; ++j) {
            stream_t st;
            stream_init(&st, (uint64_t)j, (first + (uint64_t)b) | EMIT_TAG, stream, k0, k1);
            double p[3];
            if (kind == 0) {
                const double t = 2.0 * stream_uniform(&st) - 1.0;
                const double ph = 2.0 * M_PI * stream_uniform(&st);
                const double u = r * cbrt(stream_uniform(&st));
                const double s = sqrt(1.0 - t * t);
                p[0] = u * t;
                p[1] = u * s * sin(ph);
                p[2] = u * s * cos(ph);
            } else if (kind == 1) {
                double v[3];
                if (rho[0] == 2.0 && rho[1] == 2.0 && rho[2] == 2.0) {
                    double ua = stream_uniform(&st), ub = stream_uniform(&st);
                    double rad = sqrt(-2.0 * log(1.0 - ua));
                    v[0] = rad * cos(2.0 * M_PI * ub);
                    v[1] = rad * sin(2.0 * M_PI * ub);
                    ua = stream_uniform(&st);
                    ub = stream_uniform(&st);
                    v[2] = sqrt(-2.0 * log(1.0 - ua)) * cos(2.0 * M_PI * ub);
                    for (int a = 0; a < 3; ++a) v[a] *= fwhm[a] / 2.355;
                } else {
                    for (int a = 0; a < 3; ++a) v[a] = gennorm(fwhm[a], rho[a], &st);
                }
                rot3(rot, v, p);
            } else {
                double v0, v1;
                if (rho[0] == 2.0 && rho[1] == 2.0) {
                    const double ua = stream_uniform(&st), ub = stream_uniform(&st);
                    const double rad = sqrt(-2.0 * log(1.0 - ua));
                    v0 = rad * cos(2.0 * M_PI * ub) * (fwhm[0] / 2.35);
                    v1 = rad * sin(2.0 * M_PI * ub) * (fwhm[1] / 2.35);
                } else {
                    v0 = gennorm(fwhm[0], rho[0], &st);
                    v1 = gennorm(fwhm[1], rho[1], &st);
                }
                p[0] = rot[0] * v0 + rot[1] * v1;
                p[1] = rot[3] * v0 + rot[4] * v1;
                p[2] = rot[6] * v0 + rot[7] * v1;
                const double u = stream_uniform(&st);
                if (attenuation > 0.0 && isfinite(attenuation))
                    p[2] += -log1p(u * expm1(-depth / attenuation)) * attenuation;
                else
                    p[2] += u * depth;
            }
            double *row = out + ((int64_t)b * n + j) * 4;
            row[0] = p[0];
            row[1] = p[1];
            row[2] = p[2];
            row[3] = random_phase ? 2.0 * M_PI * stream_uniform(&st) : 0.0;
        }
    }
}

/* Rotation of image b's sites: A @ rot with A per orientation (0 none,
 * 1 uniform random (Arvo, Graphics Gems III), 2 random angle about axis). */
void orc_site_rotation(int orientation, const double axis[3], const double rot[9], uint64_t k0, uint64_t k1,
                       uint64_t stream, uint64_t image, double *M) {
    double A[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    if (orientation) {
        stream_t st;
        stream_init(&st, ~0ull, image | EMIT_TAG, stream, k0, k1);
        if (orientation == 1) {
            const double th = 2.0 * M_PI * stream_uniform(&st), ph = 2.0 * M_PI * stream_uniform(&st);
            const double z = stream_uniform(&st);
            const double V[3] = {cos(ph) * sqrt(z), sin(ph) * sqrt(z), sqrt(1.0 - z)};
            const double R[9] = {cos(th), sin(th), 0.0, -sin(th), cos(th), 0.0, 0.0, 0.0, 1.0};
            double H[9];
            for (int i = 0; i < 3; ++i)
                for (int k = 0; k < 3; ++k) H[3 * i + k] = 2.0 * V[i] * V[k] - (i == k ? 1.0 : 0.0);
            for (int i = 0; i < 3; ++i)
                for (int k = 0; k < 3; ++k) A[3 * i + k] = H[3 * i] * R[k] + H[3 * i + 1] * R[3 + k] + H[3 * i + 2] * R[6 + k];
        } else {
            const double nrm = sqrt(axis[0] * axis[0] + axis[1] * axis[1] + axis[2] * axis[2]);
            const double u[3] = {axis[0] / nrm, axis[1] / nrm, axis[2] / nrm};
            const double t = 2.0 * M_PI * stream_uniform(&st);
            const double s = sin(t), c = cos(t);
            const double K[9] = {0.0, -u[2], u[1], u[2], 0.0, -u[0], -u[1], u[0], 0.0};
            for (int i = 0; i < 3; ++i)
                for (int k = 0; k < 3; ++k) A[3 * i + k] = (i == k ? c : 0.0) + s * K[3 * i + k] + (1.0 - c) * u[i] * u[k];
        }
    }
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) M[3 * i + k] = A[3 * i] * rot[k] + A[3 * i + 1] * rot[3 + k] + A[3 * i + 2] * rot[6 + k];
}

typedef struct {
    double key;
    int64_t idx;
} keyed_t;

static int cmp_keyed(const void *a, const void *b) {
    const keyed_t *x = (const keyed_t *)a, *y = (const keyed_t *)b;
    if (x->key < y->key) return -1;
    if (x->key > y->key) return 1;
    return (x->idx > y->idx) - (x->idx < y->idx);
}

static int cmp_i64(const void *a, const void *b) {
    const int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    return (x > y) - (x < y);
}

/* Lattice-site subsample; out (n_images * n, 4); selected (optional,
 * n_images * n) receives the site index of every row. */
void orc_emit_sites(const double *sites, int64_t m, int32_t n_images, int64_t n, int weighted, const double fwhm[3],
                    const double rho[3], int orientation, const double axis[3], const double rot[9], int random_phase,
                    uint64_t k0, uint64_t k1, uint64_t stream, uint64_t first, double *out, int64_t *selected) {
    keyed_t *keys = (keyed_t *)malloc(sizeof(keyed_t) * (size_t)m);
    int64_t *pick = (int64_t *)malloc(sizeof(int64_t) * (size_t)m);
    double s[3];
    for (int a = 0; a < 3; ++a) s[a] = weighted ? log(2.0) * pow(2.0 / fwhm[a], rho[a]) : 0.0;
    for (int32_t b = 0; b < n_images; ++b) {
        const uint64_t img = first + (uint64_t)b;
        double M[9];
        orc_site_rotation(orientation, axis, rot, k0, k1, stream, img, M);
        for (int64_t base = 0, round = 0; base < n; base += m, ++round) {
            const int64_t take = n - base < m ? n - base : m;
            const uint64_t tag = img | SITE_TAG | ((uint64_t)round << 44);
            for (int64_t i = 0; i < m; ++i) {
                const uint64_t ctr[4] = {1, (uint64_t)i, tag, stream};
                const uint64_t key[2] = {k0, k1};
                uint64_t w[4];
                philox4x64(ctr, key, w);
                const double u = u01(w[0]);
                double kv = u;
                if (weighted) {
                    double x[3];
                    rot3(M, sites + 3 * i, x);
                    double e = 0.0;
                    for (int a = 0; a < 3; ++a) {
                        const double ax = fabs(x[a]);
                        e += (rho[a] == 2.0 ? ax * ax : pow(ax, rho[a])) * s[a];
                    }
                    const double wt = exp(-e);
                    kv = wt > 0.0 ? -log1p(-u) / wt : INFINITY;
                }
                keys[i].key = kv;
                keys[i].idx = i;
            }
            qsort(keys, (size_t)m, sizeof(keyed_t), cmp_keyed);
            for (int64_t t = 0; t < take; ++t) pick[t] = keys[t].idx;
            qsort(pick, (size_t)take, sizeof(int64_t), cmp_i64);
            for (int64_t t = 0; t < take; ++t) {
                const int64_t j = base + t;
                double *row = out + ((int64_t)b * n + j) * 4;
                rot3(M, sites + 3 * pick[t], row);
                double phase = 0.0;
                if (random_phase) {
                    stream_t st;
                    stream_init(&st, (uint64_t)j, img | EMIT_TAG, stream, k0, k1);
                    phase = 2.0 * M_PI * stream_uniform(&st);
                }
                row[3] = phase;
                if (selected) selected[(int64_t)b * n + j] = pick[t];
            }
        }
    }
    free(keys);
    free(pick);
}

/* Envelope weight of every site (the crystal's fwhm weighting before
 * normalisation, simobj.py:463-476, with |x| for the power). */
void orc_site_weights(const double *sites, int64_t m, const double M[9], const double fwhm[3], const double rho[3],
                      double *w) {
    double s[3];
    for (int a = 0; a < 3; ++a) s[a] = log(2.0) * pow(2.0 / fwhm[a], rho[a]);
    for (int64_t i = 0; i < m; ++i) {
        double x[3];
        rot3(M, sites + 3 * i, x);
        double e = 0.0;
        for (int a = 0; a < 3; ++a) {
            const double ax = fabs(x[a]);
            e += (rho[a] == 2.0 ? ax * ax : pow(ax, rho[a])) * s[a];
        }
        w[i] = exp(-e);
    }
}
