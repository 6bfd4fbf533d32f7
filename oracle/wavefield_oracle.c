/*
 * ORACLE — test infrastructure only.
 *
 * CPU restatement (plain C, FP64, OpenMP over detector rows) of the reference's
 * emitter-wavefield direct sum and of its time-dependent variant.  It is the
 * checker for the CUDA library in idi_b200/csrc: the parity tests, smoke() and
 * the CPU-baseline leg of bench.py call it; the product never does.
 *
 * Reference algorithm followed (paths inside the idi project):
 *   pixel position        idi/simulation/cpu.py:76-80
 *   far-field q, phase    idi/simulation/cpu.py:57-66, 85-89
 *   near-field phase      idi/simulation/cpu.py:42-55
 *   Kahan complex sum     idi/simulation/cpu.py:91-107
 *   second-order term     idi/simulation/sim.cu:88 (the GPU-only "secondorder" setting)
 *   time-dependent path   idi/simulation/time.py:7-45 (_decaysum, _psort, _integral),
 *                         idi/simulation/time.py:48-98 (simulate), far field
 *   near-field arrival    idi/simulation/simtime.cu:50-83 (trans1nf)
 *
 * Rounding sequence.  The reference CPU kernel is compiled by numba with
 * fastmath {contract, arcp, ninf, nnan}; LLVM contracts its multiply-adds into
 * FMAs in a fixed pattern.  That pattern was identified by recovering the
 * phase of single-emitter runs of the reference (atan2 of its output) and
 * comparing it bit for bit with candidate sequences; the sequences below are
 * the ones that matched on every probe:
 *   near field  dist  = sqrt(fma(c, c, fma(a, a, b*b)))   a,b,c = det - atom
 *               phase = fma((dist - detz) + z, k, psi)
 *   far field   phase = -fma(z, qz, fma(x, qx, y*qy)) + psi
 *   rotation    M @ v  row i = fma(M[i,2], v2, fma(M[i,0], v0, M[i,1]*v1))
 * and for time.py (numpy / OpenBLAS):
 *   np.inner    s     = fma(q2, z, fma(q1, y, q0*x))
 *   dets @ M.T  row   = fma(M[i,2], v2, fma(M[i,1], v1, M[i,0]*v0))
 * This file is compiled with -ffp-contract=off so that only the fma() calls
 * written here fuse.
 *
 * Extensions that have no reference code (amplitudes a_j, the adjoint, the
 * accurate near-field form) are the mathematical extensions of cpu.py:42-107
 * and are marked as such where they appear.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_NF 1
#define ORC_SCALE 2
#define ORC_SECONDORDER 4
#define ORC_ACCURATE 8

typedef struct {
    int32_t nx, ny;
    double pixelsize, detz, k;
    double offx, offy;
    double rot[9];
    int32_t has_rot;
} orc_geom;

/* idi/simulation/cpu.py:76-80 (detector pixel position, float maxx/2) */
static void pixel_cpu(const orc_geom *g, int ix, int iy, double d[3]) {
    double x = (ix - g->nx / 2.0) * g->pixelsize + g->offx;
    double y = (iy - g->ny / 2.0) * g->pixelsize + g->offy;
    double z = g->detz;
    if (g->has_rot) {
        const double *M = g->rot;
        d[0] = fma(M[2], z, fma(M[0], x, M[1] * y));
        d[1] = fma(M[5], z, fma(M[3], x, M[4] * y));
        d[2] = fma(M[8], z, fma(M[6], x, M[7] * y));
    } else {
        d[0] = x; d[1] = y; d[2] = z;
    }
}

/*
 * Forward direct sum for one image: out[2*(ix*ny+iy)+{0,1}] = Re/Im E_p.
 * atoms: (n,4) [x,y,z,psi]; amp: (n) or NULL (unit amplitudes, the reference).
 */
void orc_wavefield(const orc_geom *g, int flags, const double *atoms, const double *amp,
                   int64_t n, double *out) {
    const int nf = flags & ORC_NF, scale = flags & ORC_SCALE;
    const int second = flags & ORC_SECONDORDER, accurate = flags & ORC_ACCURATE;
    const double k = g->k;
#pragma omp parallel for schedule(dynamic, 1)
    for (int ix = 0; ix < g->nx; ix++) {
        for (int iy = 0; iy < g->ny; iy++) {
            double d[3];
            pixel_cpu(g, ix, iy, d);
            const double detx = d[0], dety = d[1], detz = d[2];
            double qx = 0, qy = 0, qz = 0, rdist = 0, c2 = 0;
            double D = 0, pconst = 0;
            if (!nf) {
                /* cpu.py:86-89 */
                rdist = 1.0 / sqrt((detx * detx + dety * dety) + detz * detz);
                qz = k * (detz * rdist - 1.0);
                qx = k * (detx * rdist);
                qy = k * (dety * rdist);
                c2 = k * rdist / 2.0; /* sim.cu:83 */
            } else if (accurate) {
                /* k (|d| - d_z) without cancellation, (dx^2+dy^2)/(|d|+d_z), and
                 * reduced mod 2pi in turns before it meets the per-emitter phase */
                D = sqrt((detx * detx + dety * dety) + detz * detz);
                const double c = k / (2.0 * M_PI) * ((detx * detx + dety * dety) / (D + detz));
                pconst = 2.0 * M_PI * (c - rint(c));
            }
            double ax = 0, ay = 0, cx = 0, cy = 0;
            for (int64_t j = 0; j < n; j++) {
                const double x = atoms[4 * j], y = atoms[4 * j + 1], z = atoms[4 * j + 2];
                const double psi = atoms[4 * j + 3];
                double phase, w = 1.0;
                if (nf) {
                    const double a = detx - x, b = dety - y, c = detz - z;
                    const double dist = sqrt(fma(c, c, fma(a, a, b * b)));
                    if (accurate) {
                        /* extension: |d-r|-|d| = (|r|^2 - 2 d.r) / (|d-r| + |d|) */
                        const double rr = (x * x + y * y) + z * z;
                        const double dr = (detx * x + dety * y) + detz * z;
                        const double delta = (rr - 2.0 * dr) / (dist + D);
                        phase = pconst + (k * (delta + z) + psi);
                    } else {
                        phase = fma((dist - detz) + z, k, psi); /* cpu.py:47 */
                    }
                    if (scale) w = 1.0 / dist; /* cpu.py:52 */
                } else {
                    phase = -fma(z, qz, fma(x, qx, y * qy)) + psi; /* cpu.py:59 */
                    if (second) phase += c2 * (x * x + y * y);  /* sim.cu:88 */
                    if (scale) w = rdist;                        /* cpu.py:64 */
                }
                if (amp) w *= amp[j];
                const double px = w * cos(phase), py = w * sin(phase);
                /* Kahan summation, cpu.py:97-105 */
                const double yx = px - cx, yy = py - cy;
                const double tx = ax + yx, ty = ay + yy;
                cx = (tx - ax) - yx;
                cy = (ty - ay) - yy;
                ax = tx;
                ay = ty;
            }
            out[2 * ((int64_t)ix * g->ny + iy)] = ax;
            out[2 * ((int64_t)ix * g->ny + iy) + 1] = ay;
        }
    }
}

/*
 * Adjoint of L = sum_p (I_p - T_p)^2 with I_p = |E_p|^2 (extension; no
 * reference code).  With G_p = 2 (I_p - T_p) conj(E_p) * 2 and e_pj = w a e^{i phi}:
 *   dL/dpsi_j = sum_p Re(G_p i e_pj) = -sum_p Im(G_p e_pj)
 *   dL/da_j   = sum_p Re(G_p w e^{i phi})
 *   dL/dr_j   = dL/dpsi-like term * grad_r phi_pj  (+ the grad of w for "scale")
 * E (2*npix) must hold the forward field of the same inputs.  Gradients are
 * written to gpos (n,3), gpsi (n), gamp (n).  Returns the loss.
 */
double orc_adjoint(const orc_geom *g, int flags, const double *atoms, const double *amp,
                   int64_t n, const double *E, const double *target, double *gpos,
                   double *gpsi, double *gamp) {
    const int nf = flags & ORC_NF, scale = flags & ORC_SCALE, second = flags & ORC_SECONDORDER;
    const double k = g->k;
    const int64_t npix = (int64_t)g->nx * g->ny;
    double *G = (double *)malloc(sizeof(double) * 2 * npix);
    double loss = 0;
    for (int64_t p = 0; p < npix; p++) {
        const double er = E[2 * p], ei = E[2 * p + 1];
        const double I = er * er + ei * ei;
        const double r = I - target[p];
        loss += r * r;
        G[2 * p] = 4.0 * r * er;
        G[2 * p + 1] = -4.0 * r * ei;
    }
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t j = 0; j < n; j++) {
        const double x = atoms[4 * j], y = atoms[4 * j + 1], z = atoms[4 * j + 2];
        const double psi = atoms[4 * j + 3];
        const double aj = amp ? amp[j] : 1.0;
        double sx = 0, sy = 0, sz = 0, sp = 0, sa = 0;
        for (int ix = 0; ix < g->nx; ix++) {
            for (int iy = 0; iy < g->ny; iy++) {
                const int64_t p = (int64_t)ix * g->ny + iy;
                double d[3];
                pixel_cpu(g, ix, iy, d);
                double phase, w = 1.0, gx, gy, gz; /* grad_r phase */
                double wx = 0, wy = 0, wz = 0;   /* grad_r w */
                if (nf) {
                    const double a = d[0] - x, b = d[1] - y, c = d[2] - z;
                    const double dist = sqrt(fma(c, c, fma(a, a, b * b)));
                    phase = fma((dist - d[2]) + z, k, psi);
                    gx = k * (-a / dist);
                    gy = k * (-b / dist);
                    gz = k * (-c / dist + 1.0);
                    if (scale) {
                        w = 1.0 / dist;
                        const double w3 = w * w * w;
                        wx = a * w3; wy = b * w3; wz = c * w3;
                    }
                } else {
                    const double rd = 1.0 / sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]);
                    const double qz = k * (d[2] * rd - 1.0), qx = k * (d[0] * rd), qy = k * (d[1] * rd);
                    phase = -fma(z, qz, fma(x, qx, y * qy)) + psi;
                    gx = -qx; gy = -qy; gz = -qz;
                    if (second) {
                        const double c2 = k * rd / 2.0;
                        phase += c2 * (x * x + y * y);
                        gx += 2.0 * c2 * x;
                        gy += 2.0 * c2 * y;
                    }
                    if (scale) w = rd;
                }
                const double cs = cos(phase), sn = sin(phase);
                /* G * e^{i phi} */
                const double zr = G[2 * p] * cs - G[2 * p + 1] * sn;
                const double zi = G[2 * p] * sn + G[2 * p + 1] * cs;
                sa += w * zr;
                const double dphi = -aj * w * zi;
                sp += dphi;
                sx += dphi * gx + aj * zr * wx;
                sy += dphi * gy + aj * zr * wy;
                sz += dphi * gz + aj * zr * wz;
            }
        }
        gpos[3 * j] = sx;
        gpos[3 * j + 1] = sy;
        gpos[3 * j + 2] = sz;
        gpsi[j] = sp;
        if (gamp) gamp[j] = sa;
    }
    free(G);
    return loss;
}

/* ---------------------------------------------------------------------- */
/* time-dependent path                                                     */
/* ---------------------------------------------------------------------- */

typedef struct {
    double t;
    int64_t i;
} orc_key;

static int key_cmp(const void *a, const void *b) {
    const orc_key *x = (const orc_key *)a, *y = (const orc_key *)b;
    if (x->t < y->t) return -1;
    if (x->t > y->t) return 1;
    return (x->i > y->i) - (x->i < y->i);
}

/* time.py:77-81 — meshgrid(...).T.reshape(-1,3): pixel index = ix*ny + iy */
static void pixel_time(const orc_geom *g, int ix, int iy, double d[3]) {
    double x = g->pixelsize * (ix - g->nx / 2.0);
    double y = g->pixelsize * (iy - g->ny / 2.0);
    double z = g->detz;
    if (g->has_rot) {
        const double *M = g->rot;
        d[0] = fma(M[2], z, fma(M[1], y, M[0] * x));
        d[1] = fma(M[5], z, fma(M[4], y, M[3] * x));
        d[2] = fma(M[8], z, fma(M[7], y, M[6] * x));
    } else {
        d[0] = x; d[1] = y; d[2] = z;
    }
}

/*
 * Per-pixel arrival keys and amplitudes (unsorted, emitter order).
 * far field  time.py:89-95   s = inner(d/|d| - z_hat, r); t = -s/c + t_j;
 *                            e = exp(-i (s k - psi)) [/|d|]
 * near field simtime.cu:58-79 (double mode)  s = |d-r| - |d| + z; t = s/c + t_j;
 *                            e = exp(i (s k + psi)) [/|d-r|]
 */
void orc_time_keys(const orc_geom *g, int flags, const double *atoms, const double *times,
                   int64_t n, double c, int ix, int iy, double *t, double *er, double *ei) {
    double d[3];
    pixel_time(g, ix, iy, d);
    const double k = g->k;
    const double dn = sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]);
    if (!(flags & ORC_NF)) {
        const double q0 = d[0] / dn, q1 = d[1] / dn, q2 = d[2] / dn - 1.0;
        for (int64_t j = 0; j < n; j++) {
            const double x = atoms[4 * j], y = atoms[4 * j + 1], z = atoms[4 * j + 2];
            const double s = fma(q2, z, fma(q1, y, q0 * x));
            const double th = -(s * k - atoms[4 * j + 3]);
            double re = cos(th), im = sin(th);
            if (flags & ORC_SCALE) { re = re / dn; im = im / dn; }
            t[j] = -s / c + times[j];
            er[j] = re;
            ei[j] = im;
        }
    } else {
        for (int64_t j = 0; j < n; j++) {
            const double x = atoms[4 * j], y = atoms[4 * j + 1], z = atoms[4 * j + 2];
            const double a = d[0] - x, b = d[1] - y, cc = d[2] - z;
            const double dist = sqrt(fma(cc, cc, fma(a, a, b * b)));
            const double s = (dist - dn) + z;
            const double th = s * k + atoms[4 * j + 3];
            double re = cos(th), im = sin(th);
            if (flags & ORC_SCALE) { re = re / dist; im = im / dist; }
            t[j] = s / c + times[j];
            er[j] = re;
            ei[j] = im;
        }
    }
}

/*
 * Sorted-order output for one pixel (index permutation), used by the
 * ordering tests: order[m] = emitter index of the m-th earliest arrival.
 * Ties (never observed) are broken by emitter index.
 */
void orc_time_order(const orc_geom *g, int flags, const double *atoms, const double *times,
                    int64_t n, double c, int ix, int iy, int64_t *order) {
    double *t = (double *)malloc(sizeof(double) * n * 3);
    orc_key *kv = (orc_key *)malloc(sizeof(orc_key) * n);
    orc_time_keys(g, flags, atoms, times, n, c, ix, iy, t, t + n, t + 2 * n);
    for (int64_t j = 0; j < n; j++) { kv[j].t = t[j]; kv[j].i = j; }
    qsort(kv, n, sizeof(orc_key), key_cmp);
    for (int64_t j = 0; j < n; j++) order[j] = kv[j].i;
    free(kv);
    free(t);
}

/* numpy's pairwise summation (unrolled by 8, block 128), for np.sum parity */
static double pairwise_sum(const double *a, int64_t n) {
    if (n < 8) {
        double res = 0.;
        for (int64_t i = 0; i < n; i++) res += a[i];
        return res;
    } else if (n <= 128) {
        double r[8];
        for (int i = 0; i < 8; i++) r[i] = a[i];
        int64_t i;
        for (i = 8; i < n - (n % 8); i += 8)
            for (int m = 0; m < 8; m++) r[m] += a[i + m];
        double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
        for (; i < n; i++) res += a[i];
        return res;
    } else {
        int64_t n2 = n / 2;
        n2 -= n2 % 8;
        return pairwise_sum(a, n2) + pairwise_sum(a + n2, n - n2);
    }
}

/*
 * Time-dependent intensity image, time.py:48-98 (far field) or the near-field
 * arrival of simtime.cu:58-79.  out: (nx*ny) float64.
 * Per pixel: sort by arrival (time.py:19-29), decaying scan (time.py:7-16),
 * integral (time.py:36-45).
 */
/*
 * Digest of one pixel's arrival order (a check on every pixel's order without
 * storing it): H = sum_m (j_m + 1) B^m mod 2^64 over the sorted emitter
 * indices j_m, B = 0x9E3779B97F4A7C15.  B = 1 mod 4, so B^d - 1 has at most
 * 2 + log2(d) factors of 2 and a transposition of two indices (differing by
 * less than 2^15 at positions less than 2^15 apart) always changes H.
 */
#define ORC_DIGEST_BASE 0x9E3779B97F4A7C15ull

void orc_time_image_digest(const orc_geom *g, int flags, const double *atoms, const double *times,
                           int64_t n, double c, double tau, double *out, uint64_t *digest, int64_t *ties);

void orc_time_image(const orc_geom *g, int flags, const double *atoms, const double *times,
                    int64_t n, double c, double tau, double *out) {
    orc_time_image_digest(g, flags, atoms, times, n, c, tau, out, NULL, NULL);
}

/* As orc_time_image, plus (when non-NULL) the order digest of every pixel and
 * the number of equal neighbouring keys per pixel (0: the order is unique, so
 * any sort -- the reference's unstable argsort included -- gives it). */
void orc_time_image_digest(const orc_geom *g, int flags, const double *atoms, const double *times,
                           int64_t n, double c, double tau, double *out, uint64_t *digest, int64_t *ties) {
#pragma omp parallel
    {
        double *buf = (double *)malloc(sizeof(double) * n * 6);
        orc_key *kv = (orc_key *)malloc(sizeof(orc_key) * n);
        double *t = buf, *er = buf + n, *ei = buf + 2 * n, *terms = buf + 3 * n;
#pragma omp for schedule(dynamic, 4)
        for (int64_t p = 0; p < (int64_t)g->nx * g->ny; p++) {
            const int ix = (int)(p / g->ny), iy = (int)(p % g->ny);
            orc_time_keys(g, flags, atoms, times, n, c, ix, iy, t, er, ei);
            for (int64_t j = 0; j < n; j++) { kv[j].t = t[j]; kv[j].i = j; }
            qsort(kv, n, sizeof(orc_key), key_cmp);
            /* _decaysum on the sorted sequence */
            double xr = er[kv[0].i], xi = ei[kv[0].i];
            double Iprev = xi * xi + xr * xr;
            for (int64_t m = 1; m < n; m++) {
                const double dt = kv[m].t - kv[m - 1].t;
                const double decay = exp(-dt / tau);
                xr = er[kv[m].i] + decay * xr;
                xi = ei[kv[m].i] + decay * xi;
                /* _integral term for interval m-1 */
                terms[m - 1] = -tau / 2 * Iprev * expm1(-2 * dt / tau);
                Iprev = xi * xi + xr * xr;
            }
            out[p] = pairwise_sum(terms, n - 1) + tau / 2 * Iprev;
            if (digest) {
                uint64_t h = 0, pw = 1;
                for (int64_t m = 0; m < n; m++) {
                    h += (uint64_t)(kv[m].i + 1) * pw;
                    pw *= ORC_DIGEST_BASE;
                }
                digest[p] = h;
            }
            if (ties) {
                int64_t eq = 0;
                for (int64_t m = 1; m < n; m++) eq += kv[m].t == kv[m - 1].t;
                ties[p] = eq;
            }
        }
        free(kv);
        free(buf);
    }
}
