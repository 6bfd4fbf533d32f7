// Detector stage on the device: Poisson photon counts (randomphotons,
// idi/simulation/common.py:11-23) and charge sharing (chargesharing,
// idi/simulation/common.py:26-67).
//
//  * photon_sum_kernel / photon_sample_kernel — per-image FP64 sum of the
//    probabilities in a fixed reduction tree, then one Poisson draw per pixel:
//    below rate 10 by inversion of a uniform from the Philox4x64-10 block of
//    the pixel's quad (4 pixels per block), above it by PTRS from the pixel's
//    own stream.  2 reads of the probabilities and one write of the counts per
//    pixel.
//  * cs_seg_kernel / cs_seg_scan_kernel / cs_start_kernel — exclusive scan of
//    the photon counts (injected positions only: photon g's row in the
//    caller's arrays).
//  * cs_tile_kernel (w <= 4) / cs_gather_kernel — every output pixel sums the
//    charge of every photon within w pixels, walking source pixels in
//    row-major order and the photons of a pixel in order: the reference's
//    scatter loop adds to each pixel in exactly that order.  The tiled kernel
//    computes each photon's charge factors once per CTA in shared memory; the
//    plain one (and the tiled one for crowded regions) recomputes them per
//    target pixel.
#include <cmath>

#include "idiwf_internal.cuh"
#include "philox.cuh"

namespace idiwf {

// ---------------------------------------------------------------------------
// Poisson sampler
// ---------------------------------------------------------------------------
constexpr double kPtrsMinRate = 10.0;
constexpr int kMaxRejections = 1000;  // acceptance is above 0.88 per trial

// Counter word 0 of the blocks that hold the inversion uniforms of pixel
// quads: block (kQuadCounter, p / 4, image, stream) gives pixel p its uniform
// in word p % 4.  Per-pixel streams count word 0 up from 1 and never reach it.
constexpr uint64_t kQuadCounter = 0x8000000000000000ull;

// Inversion for 0 < lam < kPtrsMinRate: smallest k with F(k) >= u, F
// accumulated term by term in FP64.  k = 0 (u <= exp(-lam)) is settled by an
// FP32 exponential when u is clear of exp(-lam) by a relative 2^-16, far
// above its error (< 2e-6 for |lam| < 10); otherwise the FP64 comparison
// decides, so the result is that of the FP64 loop alone.
__device__ __forceinline__ double poisson_invert(double lam, double u) {
    const double e32 = (double)__expf(-(float)lam);
    if (u < e32 * (1.0 - 0x1p-16)) return 0.0;
    double p = exp(-lam), F = p;
    double k = 0.0;
    while (u > F) {
        k += 1.0;
        p = p * lam / k;
        const double Fn = F + p;
        if (Fn == F) break;  // the tail no longer changes F: u is in the last ulp
        F = Fn;
    }
    return k;
}

// lam >= kPtrsMinRate, from the pixel's own stream.
// Returns -1 when the rejection loop ran out (never in practice).
__device__ double poisson_ptrs(double lam, PhiloxStream &st) {
    // PTRS, Hoermann (1993): transformed rejection with squeeze
    const double slam = sqrt(lam), loglam = log(lam);
    const double b = 0.931 + 2.53 * slam;
    const double a = -0.059 + 0.02483 * b;
    const double invalpha = 1.1239 + 1.1328 / (b - 3.4);
    const double vr = 0.9277 - 3.6224 / (b - 2.0);
    for (int trial = 0; trial < kMaxRejections; ++trial) {
        const double U = st.uniform() - 0.5;
        const double V = st.uniform();
        const double us = 0.5 - fabs(U);
        if (!(us > 0.0)) continue;
        const double k = floor((2.0 * a / us + b) * U + lam + 0.43);
        if (us >= 0.07 && V <= vr) return k;
        if (k < 0.0 || (us < 0.013 && V > us)) continue;
        if (log(V) + log(invalpha) - log(a / (us * us) + b) <= -lam + k * loglam - lgamma(k + 1.0)) return k;
    }
    return -1.0;
}

template <typename T>
__device__ __forceinline__ double load_real(const T *p, int64_t i) {
    return (double)p[i];
}

template <typename T>
__device__ __forceinline__ void store_count(T *p, int64_t i, double v) {
    p[i] = (T)v;
}

// ---------------------------------------------------------------------------
// photon kernels
// ---------------------------------------------------------------------------
constexpr int kSumThreads = 256;
constexpr int kSumMaxBlocks = 256;
constexpr int kSumPerThread = 8;

// Partial-sum blocks per image: a function of npix only, so the reduction
// tree (and with it the sum) does not depend on the device.
static int sum_blocks(int64_t npix) {
    const int64_t per_block = (int64_t)kSumThreads * kSumPerThread;
    return (int)std::max<int64_t>(1, std::min<int64_t>(kSumMaxBlocks, (npix + per_block - 1) / per_block));
}

// Fixed-shape tree over kSumThreads values in shared memory; result in v[0].
__device__ __forceinline__ void tree_sum(double *v) {
#pragma unroll
    for (int h = kSumThreads / 2; h > 0; h >>= 1) {
        __syncthreads();
        if ((int)threadIdx.x < h) v[threadIdx.x] += v[threadIdx.x + h];
    }
    __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(kSumThreads) photon_sum_kernel(const T *__restrict__ probs, int64_t npix, int nblk,
                                                                 double *__restrict__ partials,
                                                                 uint32_t *__restrict__ err) {
    __shared__ double v[kSumThreads];
    const int b = blockIdx.y;
    const T *img = probs + (int64_t)b * npix;
    double acc = 0.0;
    bool bad = false;
    for (int64_t i = (int64_t)blockIdx.x * kSumThreads + threadIdx.x; i < npix; i += (int64_t)nblk * kSumThreads) {
        const double x = load_real(img, i);
        bad |= !(x >= 0.0);
        acc += x;
    }
    if (bad) record_error(err, kErrValue);
    v[threadIdx.x] = acc;
    tree_sum(v);
    if (threadIdx.x == 0) partials[(int64_t)b * nblk + blockIdx.x] = v[0];
}

// Pixel p below rate kPtrsMinRate inverts word p % 4 of the Philox block
// (kQuadCounter, p / 4, image, stream); a pixel at a higher rate draws its
// PTRS trials from its own stream (p, image, stream).  QUAD: one thread per
// quad of 4 consecutive pixels, so one block serves four inversions (images
// of low mean rate); otherwise one thread per pixel, and the rare inversion
// pixel computes its quad's block itself (high mean rate: the PTRS loops then
// spread over all threads).  Both give the same counts.
// MODE kPixels: one thread per pixel, inversion and PTRS.  kQuads: one
// thread per quad, inversion only; a PTRS pixel is left to the kPtrs pass and
// raises *ptrs_flag.  kPtrs: one thread per pixel, PTRS pixels only, and only
// when *ptrs_flag is set (the quad kernel then carries no PTRS code and its
// register count stays low).
constexpr int kPixels = 0, kQuads = 1, kPtrs = 2;
template <typename TI, typename TO, int MODE>
__global__ void __launch_bounds__(kSumThreads) photon_sample_kernel(const TI *__restrict__ probs, int64_t npix,
                                                                    int nblk, const double *__restrict__ partials,
                                                                    double n_photons, uint64_t k0, uint64_t k1,
                                                                    uint64_t stream, uint64_t img0,
                                                                    TO *__restrict__ out,
                                                                    uint32_t *__restrict__ err,
                                                                    uint32_t *__restrict__ ptrs_flag) {
    constexpr bool QUAD = MODE == kQuads;
    __shared__ double v[kSumThreads];
    if (MODE == kPtrs && *(volatile uint32_t *)ptrs_flag == 0u) return;
    const int b = blockIdx.y;
    v[threadIdx.x] = (int)threadIdx.x < nblk ? partials[(int64_t)b * nblk + threadIdx.x] : 0.0;
    tree_sum(v);
    const double total = v[0];
    const double scale = n_photons / total;
    const TI *img = probs + (int64_t)b * npix;
    TO *o = out + (int64_t)b * npix;
    const uint64_t ib = img0 + (uint64_t)b;
    bool bad = false;
    if (!QUAD) {
        for (int64_t p = (int64_t)blockIdx.x * kSumThreads + threadIdx.x; p < npix;
             p += (int64_t)gridDim.x * kSumThreads) {
            const double l = load_real(img, p) * scale;
            if (MODE == kPtrs && !(l >= kPtrsMinRate && l < 0x1p62)) continue;
            double k = 0.0;
            if (MODE == kPixels && l > 0.0 && l < kPtrsMinRate) {
                uint64_t w0, w1, w2, w3;
                philox4x64(kQuadCounter, (uint64_t)(p >> 2), ib, stream, k0, k1, w0, w1, w2, w3);
                const int i = (int)(p & 3);
                k = poisson_invert(l, u01(i == 0 ? w0 : (i == 1 ? w1 : (i == 2 ? w2 : w3))));
            } else if (l >= kPtrsMinRate && l < 0x1p62) {
                PhiloxStream st((uint64_t)p, ib, stream, k0, k1);
                k = poisson_ptrs(l, st);
                if (k < 0.0) {
                    bad = true;
                    k = 0.0;
                }
            } else if (!(l == 0.0) && MODE == kPixels) {
                bad = true;
            }
            store_count(o, p, k);
        }
        if (bad) record_error(err, kErrValue);
        return;
    }
    const int64_t nquad = (npix + 3) / 4;
    for (int64_t q = (int64_t)blockIdx.x * kSumThreads + threadIdx.x; q < nquad; q += (int64_t)gridDim.x * kSumThreads) {
        const int64_t p0 = 4 * q;
        const int np = (int)(npix - p0 < 4 ? npix - p0 : 4);
        double lam[4];
        bool need = false;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            lam[i] = i < np ? load_real(img, p0 + i) * scale : 0.0;
            need |= lam[i] > 0.0 && lam[i] < kPtrsMinRate;
        }
        uint64_t w[4] = {0, 0, 0, 0};
        if (need) philox4x64(kQuadCounter, (uint64_t)q, ib, stream, k0, k1, w[0], w[1], w[2], w[3]);
        double k[4];
        bool ptrs = false;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const double l = lam[i];
            k[i] = 0.0;
            if (l > 0.0 && l < kPtrsMinRate) k[i] = poisson_invert(l, u01(w[i]));
            ptrs |= l >= kPtrsMinRate && l < 0x1p62;
            bad |= i < np && !(l >= 0.0 && l < 0x1p62);
        }
        if (ptrs) *(volatile uint32_t *)ptrs_flag = 1u;  // drawn by the kPtrs pass; all writers store 1
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (i < np) store_count(o, p0 + i, k[i]);
    }
    if (bad) record_error(err, kErrValue);
}

// ---------------------------------------------------------------------------
// charge sharing
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 256;
constexpr int kScanPerThread = 16;
constexpr int64_t kScanSeg = (int64_t)kScanThreads * kScanPerThread;

// photons in a pixel: numpy astype(int) truncates toward zero; negative or
// NaN counts are invalid
template <typename T>
__device__ __forceinline__ int64_t photon_count(const T *c, int64_t i, bool &bad) {
    const double x = (double)c[i];
    if (!(x >= 0.0) || x >= 0x1p62) {
        bad = true;
        return 0;
    }
    return (int64_t)x;
}
template <>
__device__ __forceinline__ int64_t photon_count<int64_t>(const int64_t *c, int64_t i, bool &bad) {
    const int64_t x = c[i];
    if (x < 0) {
        bad = true;
        return 0;
    }
    return x;
}
template <>
__device__ __forceinline__ int64_t photon_count<int32_t>(const int32_t *c, int64_t i, bool &bad) {
    const int32_t x = c[i];
    if (x < 0) {
        bad = true;
        return 0;
    }
    return x;
}
template <>
__device__ __forceinline__ int64_t photon_count<uint32_t>(const uint32_t *c, int64_t i, bool &) {
    return (int64_t)c[i];
}

__device__ __forceinline__ int64_t block_exclusive_scan(int64_t x, int64_t *sh, int64_t &total) {
    // Hillis-Steele over kScanThreads values (integers: exact in any order)
    sh[threadIdx.x] = x;
    __syncthreads();
#pragma unroll
    for (int d = 1; d < kScanThreads; d <<= 1) {
        const int64_t y = (int)threadIdx.x >= d ? sh[threadIdx.x - d] : 0;
        __syncthreads();
        sh[threadIdx.x] += y;
        __syncthreads();
    }
    total = sh[kScanThreads - 1];
    const int64_t incl = sh[threadIdx.x];
    __syncthreads();
    return incl - x;
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) cs_seg_kernel(const T *__restrict__ counts, int64_t n,
                                                              int64_t *__restrict__ seg_tot,
                                                              uint32_t *__restrict__ err) {
    __shared__ int64_t sh[kScanThreads];
    const int64_t base = (int64_t)blockIdx.x * kScanSeg + (int64_t)threadIdx.x * kScanPerThread;
    int64_t acc = 0;
    bool bad = false;
    for (int e = 0; e < kScanPerThread; ++e) {
        const int64_t i = base + e;
        if (i < n) acc += photon_count(counts, i, bad);
    }
    if (bad) record_error(err, kErrValue);
    int64_t total;
    block_exclusive_scan(acc, sh, total);
    if (threadIdx.x == 0) seg_tot[blockIdx.x] = total;
}

// Exclusive scan of the segment totals in place (one block; exact integers).
__global__ void __launch_bounds__(kScanThreads) cs_seg_scan_kernel(int64_t *__restrict__ seg_tot, int64_t nseg,
                                                                   int64_t n_positions, uint32_t *__restrict__ err) {
    __shared__ int64_t sh[kScanThreads];
    const int64_t per = (nseg + kScanThreads - 1) / kScanThreads;
    const int64_t lo = (int64_t)threadIdx.x * per, hi = min(lo + per, nseg);
    int64_t acc = 0;
    for (int64_t i = lo; i < hi; ++i) acc += seg_tot[i];
    int64_t total;
    int64_t run = block_exclusive_scan(acc, sh, total);
    for (int64_t i = lo; i < hi; ++i) {
        const int64_t t = seg_tot[i];
        seg_tot[i] = run;
        run += t;
    }
    if (threadIdx.x == 0 && total != n_positions) record_error(err, kErrValue);
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) cs_start_kernel(const T *__restrict__ counts, int64_t n,
                                                                const int64_t *__restrict__ seg_off,
                                                                int64_t *__restrict__ start) {
    __shared__ int64_t sh[kScanThreads];
    const int64_t base = (int64_t)blockIdx.x * kScanSeg + (int64_t)threadIdx.x * kScanPerThread;
    bool bad = false;
    int64_t c[kScanPerThread];
    int64_t acc = 0;
#pragma unroll
    for (int e = 0; e < kScanPerThread; ++e) {
        const int64_t i = base + e;
        c[e] = i < n ? photon_count(counts, i, bad) : 0;
        acc += c[e];
    }
    int64_t total;
    int64_t run = block_exclusive_scan(acc, sh, total) + seg_off[blockIdx.x];
#pragma unroll
    for (int e = 0; e < kScanPerThread; ++e) {
        const int64_t i = base + e;
        if (i < n) start[i] = run;
        run += c[e];
    }
}

struct CsParams {
    int32_t n_images, nx, ny, w;
    double c;        // 1 / (2 sqrt(2) s)
    double rs2;      // sqrt(2) s
    double ns;
    uint64_t k0, k1, stream, img0;
    int64_t n_positions;
};

// erf(c + a) + erf(c - a), a = (mu - d) / (sqrt(2) s): charge fraction (x2)
// of a Gaussian centred mu inside the pixel at offset d (common.py:57-62)
__device__ __forceinline__ double cs_factor(double mu, int d, const CsParams &P) {
    const double a = (mu - (double)d) / P.rs2;
    return erf(P.c + a) + erf(P.c - a);
}

// Offsets and charge scale of photon i of source pixel q (image b), from the
// injected arrays or the photon's stream; false when an injected row is
// missing (count mismatch).
template <bool INJ>
__device__ __forceinline__ bool cs_photon(const CsParams &P, const double *__restrict__ positions,
                                          const double *__restrict__ scales, const int64_t *__restrict__ start,
                                          int64_t gq, int64_t q, int b, int64_t i, double &mux, double &muy,
                                          double &sc) {
    sc = 1.0;
    if (INJ) {
        const int64_t g = start[gq] + i;
        if (g >= P.n_positions) return false;
        mux = positions[2 * g];
        muy = positions[2 * g + 1];
        if (P.ns > 0.0 && scales) sc = scales[g];
    } else {
        uint64_t w0, w1, w2, w3;
        philox4x64((uint64_t)i + 1, (uint64_t)q, (P.img0 + (uint64_t)b) | (1ull << 63), P.stream, P.k0, P.k1, w0, w1,
                   w2, w3);
        mux = u01(w0) - 0.5;
        muy = u01(w1) - 0.5;
        if (P.ns > 0.0) sc = 1.0 + box_muller(u01(w2), u01(w3)) * P.ns;
    }
    return true;
}

// Charge deposited into output pixel (r, col) of image b: source pixels in
// row-major order, photons of a pixel in order (the reference's addition
// order for this pixel).
template <typename T, bool INJ>
__device__ double cs_pixel(const T *__restrict__ counts, const CsParams &P, const double *__restrict__ positions,
                           const double *__restrict__ scales, const int64_t *__restrict__ start, int b, int r,
                           int col, bool &bad) {
    const int64_t npix = (int64_t)P.nx * P.ny;
    double acc = 0.0;
    const int r0 = max(r - P.w, 0), r1 = min(r + P.w, P.nx - 1);
    const int c0 = max(col - P.w, 0), c1 = min(col + P.w, P.ny - 1);
    for (int qr = r0; qr <= r1; ++qr) {
        const int dr = r - qr;
        for (int qc = c0; qc <= c1; ++qc) {
            const int dc = col - qc;
            const int64_t q = (int64_t)qr * P.ny + qc;
            const int64_t gq = (int64_t)b * npix + q;
            const int64_t n = photon_count(counts, gq, bad);
            for (int64_t i = 0; i < n; ++i) {
                double mux, muy, sc;
                if (!cs_photon<INJ>(P, positions, scales, start, gq, q, b, i, mux, muy, sc)) {
                    bad = true;
                    break;
                }
                // k[x, y] = (1/4 f_x) f_y, deposited at (hit_x + y - w, hit_y + x - w)
                const double kxy = (0.25 * cs_factor(mux, dc, P)) * cs_factor(muy, dr, P);
                acc += P.ns > 0.0 ? sc * kxy : kxy;
            }
        }
    }
    return acc;
}

template <typename T, bool INJ>
__global__ void __launch_bounds__(256) cs_gather_kernel(const T *__restrict__ counts, const CsParams P,
                                                        const double *__restrict__ positions,
                                                        const double *__restrict__ scales,
                                                        const int64_t *__restrict__ start,
                                                        double *__restrict__ out, uint32_t *__restrict__ err) {
    const int64_t npix = (int64_t)P.nx * P.ny;
    const int64_t total = npix * P.n_images;
    bool bad = false;
    for (int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; o < total; o += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(o / npix);
        const int64_t po = o - (int64_t)b * npix;
        const int r = (int)(po / P.ny), col = (int)(po - (int64_t)r * P.ny);
        out[o] = cs_pixel<T, INJ>(counts, P, positions, scales, start, b, r, col, bad);
    }
    if (bad) record_error(err, kErrValue);
}

// Tiled gather: a CTA owns a kCsTR x kCsTC tile of output pixels.  It stages
// the counts of the tile and its w-pixel halo, numbers the region's photons
// (exclusive scan), computes each photon's 2 (2w + 1) charge factors once,
// and every output pixel then sums over its neighbours' photons from those
// factors -- the same products in the same order as cs_pixel.  A region with
// more photons than the shared memory holds takes cs_pixel.
constexpr int kCsTR = 8, kCsTC = 32, kCsMaxW = 4;
constexpr size_t kCsFactorBytes = 64 * 1024;

template <typename T, bool INJ>
__global__ void __launch_bounds__(256) cs_tile_kernel(const T *__restrict__ counts, const CsParams P,
                                                      const double *__restrict__ positions,
                                                      const double *__restrict__ scales,
                                                      const int64_t *__restrict__ start, double *__restrict__ out,
                                                      uint32_t *__restrict__ err, int cap) {
    extern __shared__ __align__(16) double csm[];
    __shared__ int wsum[8];
    __shared__ int s_total;
    const int w = P.w, KW = 2 * w + 1;
    const int RH = kCsTR + 2 * w, RW = kCsTC + 2 * w, RN = RH * RW;
    double *fx = csm;
    double *fy = fx + (size_t)cap * KW;
    double *scl = fy + (size_t)cap * KW;
    double *mu = scl + cap;  // (mu_x, mu_y) per photon
    int *rc = reinterpret_cast<int *>(mu + 2 * (size_t)cap);
    int *rs = rc + RN;
    const int64_t npix = (int64_t)P.nx * P.ny;
    const int b = blockIdx.z;
    const int r0 = blockIdx.y * kCsTR, c0 = blockIdx.x * kCsTC;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    bool bad = false;
    for (int ri = tid; ri < RN; ri += blockDim.x) {
        const int gr = r0 - w + ri / RW, gc = c0 - w + ri % RW;
        int n = 0;
        if (gr >= 0 && gr < P.nx && gc >= 0 && gc < P.ny)
            n = (int)min(photon_count(counts, (int64_t)b * npix + (int64_t)gr * P.ny + gc, bad), (int64_t)1 << 24);
        rc[ri] = n;
    }
    __syncthreads();
    // exclusive scan of the region's counts (RN <= 16 x 40 < 3 per thread)
    const int E = (RN + blockDim.x - 1) / blockDim.x;
    const int e0 = tid * E, e1 = min(e0 + E, RN);
    int sum = 0;
    for (int e = e0; e < e1; ++e) sum = min(sum + rc[e], 1 << 28);
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl = min(incl + y, 1 << 28);
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    int run = incl - sum;
    for (int v = 0; v < warp; ++v) run = min(run + wsum[v], 1 << 28);
    for (int e = e0; e < e1; ++e) {
        rs[e] = run;
        run = min(run + rc[e], 1 << 28);
    }
    if (tid == blockDim.x - 1) s_total = run;
    __syncthreads();
    const int r = r0 + tid / kCsTC, col = c0 + tid % kCsTC;
    const bool inside = r < P.nx && col < P.ny;
    if (s_total > cap) {  // uniform across the CTA
        if (inside) out[(int64_t)b * npix + (int64_t)r * P.ny + col] =
            cs_pixel<T, INJ>(counts, P, positions, scales, start, b, r, col, bad);
    } else {
        // the photons' offsets and scales, then their factors, one (photon,
        // factor) item per thread so the erf work spreads over the CTA
        for (int ri = tid; ri < RN; ri += blockDim.x) {
            const int n = rc[ri];
            if (n == 0) continue;
            const int gr = r0 - w + ri / RW, gc = c0 - w + ri % RW;
            const int64_t q = (int64_t)gr * P.ny + gc, gq = (int64_t)b * npix + q;
            for (int i = 0; i < n; ++i) {
                const int slot = rs[ri] + i;
                double mux = 0.0, muy = 0.0, sc = 1.0;
                if (!cs_photon<INJ>(P, positions, scales, start, gq, q, b, i, mux, muy, sc)) {
                    bad = true;
                    sc = 0.0;
                }
                mu[2 * slot] = mux;
                mu[2 * slot + 1] = muy;
                scl[slot] = sc;
            }
        }
        __syncthreads();
        const int items = s_total * 2 * KW;
        for (int it = tid; it < items; it += blockDim.x) {
            const int slot = it / (2 * KW), f = it - slot * 2 * KW;
            if (f < KW)
                fx[(size_t)slot * KW + f] = cs_factor(mu[2 * slot], f - w, P);
            else
                fy[(size_t)slot * KW + f - KW] = cs_factor(mu[2 * slot + 1], f - KW - w, P);
        }
        __syncthreads();
        if (inside) {
            double acc = 0.0;
            const int qr0 = max(r - w, 0), qr1 = min(r + w, P.nx - 1);
            const int qc0 = max(col - w, 0), qc1 = min(col + w, P.ny - 1);
            for (int qr = qr0; qr <= qr1; ++qr) {
                const int dr = r - qr;
                for (int qc = qc0; qc <= qc1; ++qc) {
                    const int dc = col - qc;
                    const int ri = (qr - (r0 - w)) * RW + (qc - (c0 - w));
                    const int n = rc[ri], base = rs[ri];
                    for (int i = 0; i < n; ++i) {
                        const int sl = base + i;
                        const double kxy = (0.25 * fx[(size_t)sl * KW + dc + w]) * fy[(size_t)sl * KW + dr + w];
                        acc += P.ns > 0.0 ? scl[sl] * kxy : kxy;
                    }
                }
            }
            out[(int64_t)b * npix + (int64_t)r * P.ny + col] = acc;
        }
    }
    if (bad) record_error(err, kErrValue);
}

// s <= 0: counts * (1 + ns N(0,1)) per pixel (common.py:35-39)
template <typename T, bool INJ>
__global__ void cs_noshare_kernel(const T *__restrict__ counts, const CsParams P, const double *__restrict__ scales,
                                  double *__restrict__ out) {
    const int64_t npix = (int64_t)P.nx * P.ny;
    const int64_t total = npix * P.n_images;
    for (int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; o < total; o += (int64_t)gridDim.x * blockDim.x) {
        const double x = (double)counts[o];
        if (!(P.ns != 0.0)) {
            out[o] = x;
            continue;
        }
        double f;
        if (INJ) {
            f = scales[o];
        } else {
            const int b = (int)(o / npix);
            const int64_t p = o - (int64_t)b * npix;
            uint64_t w0, w1, w2, w3;
            philox4x64(1, (uint64_t)p, (P.img0 + (uint64_t)b) | (1ull << 62), P.stream, P.k0, P.k1, w0, w1, w2,
                       w3);
            f = 1.0 + P.ns * box_muller(u01(w0), u01(w1));
        }
        out[o] = x * f;
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static int dev_sms() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

static size_t photons_ws_bytes(int32_t n_images, int64_t npix) {
    return 256 + align256((size_t)n_images * sum_blocks(npix) * sizeof(double));
}

template <typename TI, typename TO>
static idiwf_status launch_photons(const void *probs, int32_t n_images, int64_t npix, double n_photons,
                                   const idiwf_rng *rng, void *out, void *ws, cudaStream_t stream) {
    WsHeader *hdr = static_cast<WsHeader *>(ws);
    double *partials = reinterpret_cast<double *>(static_cast<char *>(ws) + 256);
    const int nblk = sum_blocks(npix);
    photon_sum_kernel<TI><<<dim3(nblk, n_images), kSumThreads, 0, stream>>>(static_cast<const TI *>(probs), npix,
                                                                            nblk, partials, &hdr->error);
    IDIWF_CUDA_CHECK(cudaGetLastError());
    // mean rate below 1: one thread per pixel quad (one Philox block per four
    // inversions), then a PTRS pass that returns at once when no pixel needs
    // it; above: one thread per pixel (the PTRS loops dominate)
    const bool quad = n_photons < (double)npix;
    uint32_t *flag = &hdr->work_counter;
    auto launch = [&](auto fn, int64_t items) -> idiwf_status {
        const int64_t want = (items + kSumThreads - 1) / kSumThreads;
        const int gx =
            (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)8 * dev_sms() / std::max(1, n_images) + 1));
        fn<<<dim3(gx, n_images), kSumThreads, 0, stream>>>(static_cast<const TI *>(probs), npix, nblk, partials,
                                                           n_photons, rng->key[0], rng->key[1], rng->stream,
                                                           rng->first_image, static_cast<TO *>(out), &hdr->error, flag);
        IDIWF_CUDA_CHECK(cudaGetLastError());
        return IDIWF_OK;
    };
    if (!quad) return launch(photon_sample_kernel<TI, TO, kPixels>, npix);
    IDIWF_CUDA_CHECK(cudaMemsetAsync(flag, 0, sizeof(uint32_t), stream));
    idiwf_status st = launch(photon_sample_kernel<TI, TO, kQuads>, (npix + 3) / 4);
    if (st != IDIWF_OK) return st;
    return launch(photon_sample_kernel<TI, TO, kPtrs>, npix);
}

template <typename TI>
static idiwf_status photons_out(int32_t out_dtype, const void *probs, int32_t n_images, int64_t npix,
                                double n_photons, const idiwf_rng *rng, void *out, void *ws, cudaStream_t stream) {
    switch (out_dtype) {
        case IDIWF_F64: return launch_photons<TI, double>(probs, n_images, npix, n_photons, rng, out, ws, stream);
        case IDIWF_F32: return launch_photons<TI, float>(probs, n_images, npix, n_photons, rng, out, ws, stream);
        case IDIWF_I32: return launch_photons<TI, int32_t>(probs, n_images, npix, n_photons, rng, out, ws, stream);
        case IDIWF_U32: return launch_photons<TI, uint32_t>(probs, n_images, npix, n_photons, rng, out, ws, stream);
        case IDIWF_I64: return launch_photons<TI, int64_t>(probs, n_images, npix, n_photons, rng, out, ws, stream);
        default: return set_error(IDIWF_ERR_INVALID_ARGUMENT, "out_dtype must be IDIWF_F64/F32/I32/U32/I64");
    }
}

template <typename T, bool INJ>
static idiwf_status launch_cs_gather(const T *counts, const CsParams &P, const double *positions,
                                     const double *scales, const int64_t *start, double *out, WsHeader *hdr,
                                     int blocks, cudaStream_t stream) {
    if (P.w <= kCsMaxW && P.n_images <= 65535) {
        const int KW = 2 * P.w + 1;
        const int RN = (kCsTR + 2 * P.w) * (kCsTC + 2 * P.w);
        const int cap = (int)(kCsFactorBytes / ((2 * (size_t)KW + 3) * sizeof(double)));
        const size_t smem = (size_t)cap * (2 * KW + 3) * sizeof(double) + 2 * (size_t)RN * sizeof(int);
        IDIWF_CUDA_CHECK(cudaFuncSetAttribute(cs_tile_kernel<T, INJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)smem));
        const dim3 grid((P.ny + kCsTC - 1) / kCsTC, (P.nx + kCsTR - 1) / kCsTR, P.n_images);
        cs_tile_kernel<T, INJ><<<grid, kCsTR * kCsTC, smem, stream>>>(counts, P, positions, scales, start, out,
                                                                       &hdr->error, cap);
    } else {
        cs_gather_kernel<T, INJ><<<blocks, 256, 0, stream>>>(counts, P, positions, scales, start, out, &hdr->error);
    }
    IDIWF_CUDA_CHECK(cudaGetLastError());
    return IDIWF_OK;
}

static size_t cs_ws_bytes(int32_t n_images, int32_t nx, int32_t ny, int32_t injected) {
    const int64_t n = (int64_t)n_images * nx * ny;
    const int64_t nseg = (n + kScanSeg - 1) / kScanSeg;
    size_t bytes = 256;
    if (injected) bytes += align256((size_t)nseg * 8) + align256((size_t)n * 8);
    return bytes;
}

template <typename T>
static idiwf_status launch_cs(const void *counts_v, int32_t n_images, int32_t nx, int32_t ny, double s, double ns,
                              const idiwf_rng *rng, const double *positions, const double *scales,
                              int64_t n_positions, double *out, void *ws, cudaStream_t stream) {
    const T *counts = static_cast<const T *>(counts_v);
    WsHeader *hdr = static_cast<WsHeader *>(ws);
    const int64_t n = (int64_t)n_images * nx * ny;
    CsParams P{};
    P.n_images = n_images;
    P.nx = nx;
    P.ny = ny;
    P.ns = ns;
    P.k0 = rng ? rng->key[0] : 0;
    P.k1 = rng ? rng->key[1] : 0;
    P.stream = rng ? rng->stream : 0;
    P.img0 = rng ? rng->first_image : 0;
    P.n_positions = n_positions;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)16 * dev_sms()));
    if (!(s > 0.0)) {
        if (ns != 0.0 && scales != nullptr)
            cs_noshare_kernel<T, true><<<blocks, 256, 0, stream>>>(counts, P, scales, out);
        else
            cs_noshare_kernel<T, false><<<blocks, 256, 0, stream>>>(counts, P, nullptr, out);
        IDIWF_CUDA_CHECK(cudaGetLastError());
        return IDIWF_OK;
    }
    P.w = (int)std::ceil(2.0 * s);
    P.c = 1.0 / (2.0 * std::sqrt(2.0) * s);
    P.rs2 = std::sqrt(2.0) * s;
    if (positions) {
        const int64_t nseg = (n + kScanSeg - 1) / kScanSeg;
        int64_t *seg = reinterpret_cast<int64_t *>(static_cast<char *>(ws) + 256);
        int64_t *start = reinterpret_cast<int64_t *>(static_cast<char *>(ws) + 256 + align256((size_t)nseg * 8));
        cs_seg_kernel<T><<<(unsigned)nseg, kScanThreads, 0, stream>>>(counts, n, seg, &hdr->error);
        cs_seg_scan_kernel<<<1, kScanThreads, 0, stream>>>(seg, nseg, n_positions, &hdr->error);
        cs_start_kernel<T><<<(unsigned)nseg, kScanThreads, 0, stream>>>(counts, n, seg, start);
        return launch_cs_gather<T, true>(counts, P, positions, scales, start, out, hdr, blocks, stream);
    }
    return launch_cs_gather<T, false>(counts, P, nullptr, nullptr, nullptr, out, hdr, blocks, stream);
}

}  // namespace idiwf

using namespace idiwf;

extern "C" size_t idiwf_photons_workspace_size(int32_t n_images, int64_t npix) {
    if (n_images <= 0 || npix <= 0) return 0;
    return photons_ws_bytes(n_images, npix);
}

extern "C" idiwf_status idiwf_photons(const void *probs, int32_t probs_dtype, int32_t n_images, int64_t npix,
                                      double n_photons, const idiwf_rng *rng, void *out, int32_t out_dtype,
                                      void *workspace, size_t workspace_bytes, cudaStream_t stream) {
    if (n_images <= 0 || npix <= 0) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "n_images and npix must be positive");
    if (n_images > 65535) return set_error(IDIWF_ERR_UNSUPPORTED, "at most 65535 images per call");
    if (!probs || !out || !rng) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "probs, out and rng must be non-NULL");
    if (!std::isfinite(n_photons) || n_photons < 0)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "n_photons must be finite and >= 0");
    if (!workspace || workspace_bytes < photons_ws_bytes(n_images, npix))
        return set_error(IDIWF_ERR_WORKSPACE, "workspace smaller than idiwf_photons_workspace_size()");
    if (reinterpret_cast<uintptr_t>(workspace) & 255)
        return set_error(IDIWF_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    IDIWF_CUDA_CHECK(cudaMemsetAsync(workspace, 0, 2 * sizeof(uint32_t), stream));
    if (probs_dtype == IDIWF_F64)
        return photons_out<double>(out_dtype, probs, n_images, npix, n_photons, rng, out, workspace, stream);
    if (probs_dtype == IDIWF_F32)
        return photons_out<float>(out_dtype, probs, n_images, npix, n_photons, rng, out, workspace, stream);
    return set_error(IDIWF_ERR_INVALID_ARGUMENT, "probs_dtype must be IDIWF_F64 or IDIWF_F32");
}

extern "C" size_t idiwf_chargesharing_workspace_size(int32_t n_images, int32_t nx, int32_t ny, int32_t injected) {
    if (n_images <= 0 || nx <= 0 || ny <= 0) return 0;
    return cs_ws_bytes(n_images, nx, ny, injected);
}

extern "C" idiwf_status idiwf_chargesharing(const void *counts, int32_t counts_dtype, int32_t n_images, int32_t nx,
                                            int32_t ny, double s, double ns, const idiwf_rng *rng,
                                            const double *positions, const double *scales, int64_t n_positions,
                                            double *out, void *workspace, size_t workspace_bytes,
                                            cudaStream_t stream) {
    if (n_images <= 0 || nx <= 0 || ny <= 0)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "n_images, nx and ny must be positive");
    if (!counts || !out) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "counts and out must be non-NULL");
    if (!std::isfinite(s) || !std::isfinite(ns)) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "s and ns must be finite");
    if (s > 0.0 && std::ceil(2.0 * s) > 64.0) return set_error(IDIWF_ERR_UNSUPPORTED, "s above 32 pixels");
    const bool injected = positions != nullptr && s > 0.0;
    // draws come from rng unless injected: positions (+ scales when ns > 0)
    // for s > 0, per-pixel scales for s <= 0
    const bool random = s > 0.0 ? !injected : (ns != 0.0 && scales == nullptr);
    if (random && !rng) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "rng must be non-NULL without injected draws");
    if (injected && n_positions < 0) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "n_positions must be >= 0");
    if (injected && ns > 0.0 && !scales)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "injected positions with ns > 0 need injected scales");
    if (!workspace || workspace_bytes < cs_ws_bytes(n_images, nx, ny, injected))
        return set_error(IDIWF_ERR_WORKSPACE, "workspace smaller than idiwf_chargesharing_workspace_size()");
    if (reinterpret_cast<uintptr_t>(workspace) & 255)
        return set_error(IDIWF_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    IDIWF_CUDA_CHECK(cudaMemsetAsync(workspace, 0, 2 * sizeof(uint32_t), stream));
    const double *pos = s > 0.0 ? positions : nullptr;
    switch (counts_dtype) {
        case IDIWF_F64:
            return launch_cs<double>(counts, n_images, nx, ny, s, ns, rng, pos, scales, n_positions, out, workspace, stream);
        case IDIWF_F32:
            return launch_cs<float>(counts, n_images, nx, ny, s, ns, rng, pos, scales, n_positions, out, workspace, stream);
        case IDIWF_I32:
            return launch_cs<int32_t>(counts, n_images, nx, ny, s, ns, rng, pos, scales, n_positions, out, workspace, stream);
        case IDIWF_U32:
            return launch_cs<uint32_t>(counts, n_images, nx, ny, s, ns, rng, pos, scales, n_positions, out, workspace, stream);
        case IDIWF_I64:
            return launch_cs<int64_t>(counts, n_images, nx, ny, s, ns, rng, pos, scales, n_positions, out, workspace, stream);
        default: return set_error(IDIWF_ERR_INVALID_ARGUMENT, "counts_dtype must be IDIWF_F64/F32/I32/U32/I64");
    }
}
