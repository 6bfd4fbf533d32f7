/*
 * ORACLE -- test infrastructure only.
 *
 * CPU restatement of the reference's direct q-space correlators, pair set,
 * binning and run accumulation as their kernels execute them, in FP32
 * without contraction (the build passes -ffp-contract=off):
 *  - orc_qcorr_radial: idi/reconstruction/cucorrad.py:54-116 -- one run per
 *    (reference row, row offset in [0, qmax), column offset in [-qmax, qmax]);
 *    the run starts at bin (column offset + qmax) / 2 with an empty sum, is
 *    added when the bin changes and at the end only if the last pair's bin
 *    is below qmax; bins 0..qmax-1 are returned.
 *  - orc_qcorr_3d: idi/reconstruction/cucor.py:55-104 -- the pairs of
 *    (reference row, row offset in [0, qmax), column offset in
 *    (-qmax, qmax)) and their bins, pairs binned outside the array dropped
 *    (the reference writes them out of bounds), then the assemble step's
 *    symmetrisation over the x extent of its launch, each mirror pair once.
 *    The reference adds every pair to FP32 bins; this restatement, like the
 *    device kernel, adds FP32 runs of equal-bin pairs to FP64 bins, so the
 *    two agree to FP32 rounding.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* images (n_images, nr, nc); q (nr * nc, 4); out (n_images, qmax) */
void orc_qcorr_radial(const float *q, const float *images, int32_t n_images, int32_t nr, int32_t nc, int32_t qmax,
                      double *out) {
    double *hist = (double *)malloc(sizeof(double) * (size_t)(qmax + 1));
    for (int32_t b = 0; b < n_images; ++b) {
        const float *v = images + (int64_t)b * nr * nc;
        memset(hist, 0, sizeof(double) * (size_t)(qmax + 1));
        for (int refr = 0; refr < nr; ++refr)
            for (int dr = 0; dr < qmax; ++dr) {
                const int tr = refr + dr;
                if (tr >= nr) break;
                for (int tid = 0; tid <= 2 * qmax; ++tid) {
                    const int offsetc = tid - qmax;
                    float val = 0.0f;
                    int dqold = tid / 2, dq = qmax + 1;
                    for (int refc = 0; refc < nc; ++refc) {
                        const int tc = refc + offsetc;
                        if (tc < 0 || tc >= nc) continue;
                        const float *a = q + 4 * ((int64_t)refr * nc + refc);
                        const float *t = q + 4 * ((int64_t)tr * nc + tc);
                        const float dx = a[0] - t[0], dy = a[1] - t[1], dz = a[2] - t[2];
                        const float d2 = dx * dx + dy * dy + dz * dz;
                        dq = (int)rintf(sqrtf(d2));
                        if (dq <= qmax) {
                            if (dq != dqold) {
                                hist[dqold] += (double)val;
                                dqold = dq;
                                val = 0.0f;
                            }
                            val = val + v[(int64_t)refr * nc + refc] * v[(int64_t)tr * nc + tc];
                        }
                    }
                    if (dq < qmax) hist[dq] += (double)val;
                }
            }
        for (int i = 0; i < qmax; ++i) out[(int64_t)b * qmax + i] = hist[i];
    }
    free(hist);
}

/* images (n_images, nr, nc); zd (nr, nc); out (n_images, 2 maxdqz, 2 qmax, 2 qmax) */
void orc_qcorr_3d(const float *zd, const float *images, int32_t n_images, int32_t nr, int32_t nc, int32_t qmax,
                  int32_t maxdqz, float xcenter, float ycenter, float z, double *out) {
    const int64_t D0 = 2 * (int64_t)maxdqz, D1 = 2 * (int64_t)qmax, D2 = 2 * (int64_t)qmax;
    const int64_t vol = D0 * D1 * D2;
    memset(out, 0, sizeof(double) * (size_t)(vol * n_images));
    for (int32_t b = 0; b < n_images; ++b) {
        const float *v = images + (int64_t)b * nr * nc;
        double *o = out + (int64_t)b * vol;
        for (int refr = 0; refr < nr; ++refr) {
            const float refr2 = (float)refr - xcenter;
            for (int dr = 0; dr < qmax; ++dr) {
                const int tr = refr + dr;
                if (tr >= nr) break;
                const float tr2 = (float)tr - xcenter;
                for (int offsetc = -(qmax - 1); offsetc <= qmax - 1; ++offsetc) {
                    int64_t bin = -1;
                    float val = 0.0f;
                    for (int refc = 0; refc < nc; ++refc) {
                        const int tc = refc + offsetc;
                        if (tc < 0 || tc >= nc) continue;
                        const float za = zd[(int64_t)refr * nc + refc], zb = zd[(int64_t)tr * nc + tc];
                        const int dqx = qmax + (int)rintf(tr2 * zb - refr2 * za);
                        const int dqy = qmax + (int)rintf(((float)tc - ycenter) * zb - ((float)refc - ycenter) * za);
                        const int dqz = maxdqz + (int)rintf(z * (za - zb));
                        if (dqz < 0 || dqz >= D0 || dqy < 0 || dqy >= D1 || dqx < 0 || dqx >= D2) continue;
                        const int64_t nb = ((int64_t)dqz * D1 + dqy) * D2 + dqx;
                        if (nb != bin) {
                            if (bin >= 0) o[bin] += (double)val;
                            bin = nb;
                            val = 0.0f;
                        }
                        val = val + v[(int64_t)refr * nc + refc] * v[(int64_t)tr * nc + tc];
                    }
                    if (bin >= 0) o[bin] += (double)val;
                }
            }
        }
        const int64_t n2 = D2 > 64 ? 2 * (D2 / 4) : D2 / 2;
        for (int64_t i0 = 0; i0 < D0; ++i0)
            for (int64_t i1 = 0; i1 < D1; ++i1)
                for (int64_t i2 = 0; i2 < n2; ++i2) {
                    const int64_t m0 = (D0 - i0) % D0, m1 = (D1 - i1) % D1, m2 = (D2 - i2) % D2;
                    const int64_t a = (i0 * D1 + i1) * D2 + i2, c = (m0 * D1 + m1) * D2 + m2;
                    if (a == c) {
                        o[a] = 2.0 * o[a];
                    } else if (m2 >= n2 || a < c) {
                        const double s = o[a] + o[c];
                        o[a] = s;
                        o[c] = s;
                    }
                }
    }
}
