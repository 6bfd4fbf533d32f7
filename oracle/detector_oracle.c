/*
 * ORACLE -- test infrastructure only.
 *
 * CPU restatement of the detector stage: Poisson photon counts
 * (idi/simulation/common.py:11-23 randomphotons) and charge sharing
 * (idi/simulation/common.py:26-67 chargesharing), with the random streams the
 * device library draws from.
 *
 *  - orc_philox4x64: Philox4x64-10 (Salmon et al., SC 2011).  Pinned against
 *    numpy.random.Philox's raw output by the CPU tests.
 *  - orc_photons: per-image sum in the same fixed reduction tree as the
 *    device kernel, rate = p * (n / sum) as common.py:17, and one Poisson
 *    draw per pixel: below rate 10 inversion of word p % 4 of the Philox
 *    block (2^63, p / 4, image, stream); above it PTRS (W. Hoermann 1993)
 *    from the pixel's stream (p, image, stream).
 *  - orc_chargesharing: the reference's scatter loop (common.py:49-67) --
 *    per photon, in the reference's photon order, the (2w+1)^2 kernel
 *    k[x, y] = (1/4 f_x[x]) f_y[y] added at (hit_x + y - w, hit_y + x - w) --
 *    with the photon offsets either injected or drawn from the streams the
 *    device uses.
 */
#define _DEFAULT_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "philox_oracle.h"

void orc_philox4x64(const uint64_t ctr[4], const uint64_t key[2], uint64_t out[4]) { philox4x64(ctr, key, out); }

/* Uniform doubles of one stream (counter (0, c1, c2, c3) before the first block). */
void orc_uniforms(uint64_t c1, uint64_t c2, uint64_t c3, uint64_t k0, uint64_t k1, int64_t n, double *out) {
    stream_t s;
    stream_init(&s, c1, c2, c3, k0, k1);
    for (int64_t i = 0; i < n; ++i) out[i] = stream_uniform(&s);
}

/* Inversion for 0 < lam < 10 with the uniform u of the pixel's quad block. */
static double poisson_invert(double lam, double u) {
    double p = exp(-lam), F = p, k = 0.0;
    while (u > F) {
        k += 1.0;
        p = p * lam / k;
        const double Fn = F + p;
        if (Fn == F) break;
        F = Fn;
    }
    return k;
}

/* PTRS (Hoermann 1993) for lam >= 10 from the pixel's own stream. */
static double poisson_ptrs(double lam, stream_t *st) {
    const double slam = sqrt(lam), loglam = log(lam);
    const double b = 0.931 + 2.53 * slam;
    const double a = -0.059 + 0.02483 * b;
    const double invalpha = 1.1239 + 1.1328 / (b - 3.4);
    const double vr = 0.9277 - 3.6224 / (b - 2.0);
    for (int trial = 0; trial < 1000; ++trial) {
        const double U = stream_uniform(st) - 0.5;
        const double V = stream_uniform(st);
        const double us = 0.5 - fabs(U);
        if (!(us > 0.0)) continue;
        const double k = floor((2.0 * a / us + b) * U + lam + 0.43);
        if (us >= 0.07 && V <= vr) return k;
        if (k < 0.0 || (us < 0.013 && V > us)) continue;
        int sg;
        if (log(V) + log(invalpha) - log(a / (us * us) + b) <= -lam + k * loglam - lgamma_r(k + 1.0, &sg)) return k;
    }
    return -1.0;
}

/* Sum of one image in the device's reduction tree: nblk blocks of 256
 * threads, thread t of block blk adds elements blk*256 + t + m*nblk*256 in
 * order; each block folds its 256 values pairwise (h = 128, 64, ..., 1), and
 * the nblk block sums (zero-padded to 256) are folded the same way. */
static double tree256(double *v) {
    for (int h = 128; h > 0; h >>= 1)
        for (int t = 0; t < h; ++t) v[t] += v[t + h];
    return v[0];
}

double orc_image_sum(const double *img, int64_t npix) {
    const int64_t per_block = 256 * 8;
    int64_t nblk = (npix + per_block - 1) / per_block;
    if (nblk < 1) nblk = 1;
    if (nblk > 256) nblk = 256;
    double part[256], v[256];
    for (int blk = 0; blk < 256; ++blk) part[blk] = 0.0;
    for (int64_t blk = 0; blk < nblk; ++blk) {
        for (int t = 0; t < 256; ++t) {
            double acc = 0.0;
            for (int64_t i = blk * 256 + t; i < npix; i += nblk * 256) acc += img[i];
            v[t] = acc;
        }
        part[blk] = tree256(v);
    }
    return tree256(part);
}

/* counts (B, npix) as float64; rates (optional) receives p * (n / sum). */
void orc_photons(const double *probs, int32_t n_images, int64_t npix, double n_photons, uint64_t k0, uint64_t k1,
                 uint64_t stream, uint64_t first_image, double *counts, double *rates) {
    for (int32_t b = 0; b < n_images; ++b) {
        const double *img = probs + (int64_t)b * npix;
        const double scale = n_photons / orc_image_sum(img, npix);
#pragma omp parallel for schedule(static)
        for (int64_t p = 0; p < npix; ++p) {
            const double lam = img[p] * scale;
            if (rates) rates[(int64_t)b * npix + p] = lam;
            double k = 0.0;
            if (lam > 0.0 && lam < 10.0) {
                /* block (2^63, p / 4, image, stream), word p % 4 */
                const uint64_t ctr[4] = {0x8000000000000000ull, (uint64_t)p / 4, first_image + (uint64_t)b, stream};
                const uint64_t key[2] = {k0, k1};
                uint64_t w[4];
                philox4x64(ctr, key, w);
                k = poisson_invert(lam, u01(w[p % 4]));
            } else if (lam >= 10.0 && lam < 0x1p62) {
                stream_t st;
                stream_init(&st, (uint64_t)p, first_image + (uint64_t)b, stream, k0, k1);
                k = poisson_ptrs(lam, &st);
            }
            counts[(int64_t)b * npix + p] = k;
        }
    }
}

/* Charge sharing of (B, nx, ny) integer counts into out (B, nx, ny).
 * positions: NULL (draw from the streams) or (total, 2) mu in photon order;
 * scales: per photon (s > 0) or NULL. */
void orc_chargesharing(const int64_t *counts, int32_t n_images, int32_t nx, int32_t ny, double s, double ns,
                       uint64_t k0, uint64_t k1, uint64_t stream, uint64_t first_image, const double *positions,
                       const double *scales, double *out) {
    const int64_t npix = (int64_t)nx * ny;
    const int w = (int)ceil(2.0 * s);
    const double c = 1.0 / (2.0 * sqrt(2.0) * s);
    const double rs2 = sqrt(2.0) * s;
    const int kw = 2 * w + 1;
    double *k = (double *)malloc(sizeof(double) * kw * kw);
    memset(out, 0, sizeof(double) * npix * n_images);
    int64_t g = 0;
    for (int32_t b = 0; b < n_images; ++b) {
        double *ret = out + (int64_t)b * npix;
        for (int64_t q = 0; q < npix; ++q) {
            const int hx = (int)(q / ny), hy = (int)(q % ny);
            for (int64_t i = 0; i < counts[(int64_t)b * npix + q]; ++i, ++g) {
                double mux, muy, sc = 1.0;
                if (positions) {
                    mux = positions[2 * g];
                    muy = positions[2 * g + 1];
                    if (ns > 0 && scales) sc = scales[g];
                } else {
                    const uint64_t ctr[4] = {(uint64_t)i + 1, (uint64_t)q, (first_image + (uint64_t)b) | (1ull << 63),
                                             stream};
                    const uint64_t key[2] = {k0, k1};
                    uint64_t r[4];
                    orc_philox4x64(ctr, key, r);
                    mux = u01(r[0]) - 0.5;
                    muy = u01(r[1]) - 0.5;
                    if (ns > 0) sc = 1.0 + sqrt(-2.0 * log(1.0 - u01(r[2]))) * cos(2.0 * M_PI * u01(r[3])) * ns;
                }
                for (int e = 0; e < kw * kw; ++e) k[e] = 0.25;
                for (int x = -w; x <= w; ++x) {
                    const double a = (mux - x) / rs2;
                    const double f = erf(c + a) + erf(c - a);
                    for (int y = 0; y < kw; ++y) k[(x + w) * kw + y] *= f;
                }
                for (int y = -w; y <= w; ++y) {
                    const double bb = (muy - y) / rs2;
                    const double f = erf(c + bb) + erf(c - bb);
                    for (int x = 0; x < kw; ++x) k[x * kw + (y + w)] *= f;
                }
                for (int x = 0; x < kw; ++x)
                    for (int y = 0; y < kw; ++y) {
                        const int tr = hx + y - w, tc = hy + x - w;
                        if (tr < 0 || tr >= nx || tc < 0 || tc >= ny) continue; /* charge leaves the detector */
                        ret[(int64_t)tr * ny + tc] += ns > 0 ? sc * k[x * kw + y] : k[x * kw + y];
                    }
            }
        }
    }
    free(k);
}
