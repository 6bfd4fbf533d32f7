// Forward emitter-wavefield direct sum for sm_100a.
//
// Two kernels share one persistent work-queue skeleton:
//
//  * fwd_split_kernel (IDIWF_SPLIT) — the throughput kernel.  The phase of
//    each emitter/pixel pair is formed in FP64 *in turns* with the per-pixel
//    constant part pre-folded into a magic number, so the last DFMA leaves
//    the fractional turn as 32-bit fixed point in the low word of the double
//    (phase mod 2pi for free).  Its top bit selects the half turn (folded
//    into the sign of the amplitude) and the next 23 bits become an FP32
//    angle in [-pi/2, pi/2); the near-field second-order term, sincos (MUFU), the 1/r
//    factor and the field accumulation run in FP32, two pixels per
//    instruction with Blackwell's packed f32x2 FMA.  Field sums are FP32
//    partials over 64-emitter blocks folded into Kahan-compensated totals.
//
//  * fwd_double_kernel (IDIWF_DOUBLE) — all-FP64, and op-for-op the
//    rounding sequence of the reference CPU kernel
//    (idi/simulation/cpu.py:42-107 as numba/LLVM contracts it), so its
//    fields match the reference to the last bits of sin/cos.
//
// Both stage emitter tiles from HBM to shared memory with bulk asynchronous
// copies (cp.async.bulk, mbarrier completion, double-buffered, bounded
// waits) and broadcast them to all warps; each thread owns a run of
// consecutive pixels along a detector row, so loads of the tile are
// broadcasts and the output stores are contiguous per warp.
//
// Work units are (image, pixel tile); a CTA takes units from an atomic
// counter in the workspace, images ordered by descending emitter count, so
// one launch balances a batch of images with uneven emitter counts.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <tuple>
#include <mutex>
#include <numeric>
#include <vector>

#include "idiwf_internal.cuh"

namespace idiwf {

// ---------------------------------------------------------------------------
// record layouts
// ---------------------------------------------------------------------------
// split:  r64 double4 {x, y, z, Psi}              (32 B)  Psi = magic + 1/4 + psi/2pi mod 1
//         rA  float4  {x, y, z, -w}               (16 B)  w = |r|^2 (nf) or x^2+y^2
//         rC  float   a                           ( 4 B)
//         (the kernel pairs each value with itself for the f32x2 operations;
//         storing the pairs would cost a fifth shared-memory load per emitter)
// double: r64 double4 {x, y, z, psi}, ra double a
constexpr int kSplitRecBytes = 52;
constexpr int kDoubleRecBytes = 40;
constexpr int kFold = 64;  // emitters per FP32 partial before the Kahan fold

struct SplitRecs {
    double4 *r64;
    float4 *rA;
    float *rC;
    uint32_t *rmax2;  // per image of the launch: max |r|^2 (float bits, rounded up)
};
struct DoubleRecs {
    double4 *r64;
    double *ra;
};

static inline SplitRecs split_recs(void *ws, int64_t nrec) {
    char *base = static_cast<char *>(ws) + kWsDataOffset;
    SplitRecs r;
    r.r64 = reinterpret_cast<double4 *>(base);
    base += align256(nrec * 32);
    r.rA = reinterpret_cast<float4 *>(base);
    base += align256(nrec * 16);
    r.rC = reinterpret_cast<float *>(base);
    base += align256(nrec * 4);
    r.rmax2 = reinterpret_cast<uint32_t *>(base);
    return r;
}
static inline size_t split_recs_bytes(int64_t nrec) {
    return align256(nrec * 32) + align256(nrec * 16) + align256(nrec * 4) + align256(kMaxImagesPerLaunch * 4);
}
static inline DoubleRecs double_recs(void *ws, int64_t nrec) {
    char *base = static_cast<char *>(ws) + kWsDataOffset;
    DoubleRecs r;
    r.r64 = reinterpret_cast<double4 *>(base);
    base += align256(nrec * 32);
    r.ra = reinterpret_cast<double *>(base);
    return r;
}
static inline size_t double_recs_bytes(int64_t nrec) {
    return align256(nrec * 32) + align256(nrec * 8);
}

// ---------------------------------------------------------------------------
// prep kernels: caller layout (N,4) f64 [+ amplitudes] -> padded tile records
// ---------------------------------------------------------------------------
__global__ void prep_split_kernel(const __grid_constant__ BatchParams bp, const double *__restrict__ atoms,
                                  const void *__restrict__ amps, int amp_dtype, int w_mode,
                                  double max_abs, SplitRecs rec, uint32_t *err) {
    const int b = blockIdx.y;
    const ImageDesc d = bp.img[b];
    const int64_t nrec = (int64_t)d.ntiles * bp.te;
    uint32_t r2max = 0;  // float bits; non-negative floats order like their bits
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nrec;
         j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = d.rec + j;
        if (j < d.n) {
            const int64_t s = d.src + j;
            const double4 a = reinterpret_cast<const double4 *>(atoms)[s];
            r2max = max(r2max, __float_as_uint(__double2float_ru((a.x * a.x + a.y * a.y) + a.z * a.z)));
            double psi = a.w * kInvTwoPi;
            psi = psi - rint(psi);
            // the DFMA chain of the kernel starts from this value: the magic
            // binade, +1/4 turn (bit 31 of the fixed-point phase then marks
            // the half turn centred on pi) and +2^-25 turn (rounds instead of
            // truncating to the 23 angle bits the kernel keeps)
            psi = (kTurnMagic + 0.25 + 0x1p-25) + psi;
            float amp = 1.0f;
            if (amps) amp = amp_dtype == IDIWF_F32 ? static_cast<const float *>(amps)[s]
                                                  : (float)static_cast<const double *>(amps)[s];
            if (!(fabs(a.x) <= max_abs && fabs(a.y) <= max_abs && fabs(a.z) <= max_abs))
                record_error(err, kErrRange);
            const double w = w_mode == 1 ? (a.x * a.x + a.y * a.y) + a.z * a.z
                                         : (w_mode == 2 ? a.x * a.x + a.y * a.y : 0.0);
            // w is stored negated: the kernel forms s^2 - w and subtracts h times it
            const float fx = (float)a.x, fy = (float)a.y, fz = (float)a.z, fw = (float)(-w);
            rec.r64[r] = make_double4(a.x, a.y, a.z, psi);
            rec.rA[r] = make_float4(fx, fy, fz, fw);
            rec.rC[r] = amp;
        } else {
            rec.r64[r] = make_double4(0, 0, 0, 0);
            rec.rA[r] = make_float4(0, 0, 0, 0);
            rec.rC[r] = 0.0f;
        }
    }
    // |r|_max of the image for the split kernel's pixel-run bound (the caller
    // zeroes rmax2 before the launch)
    r2max = __reduce_max_sync(0xffffffffu, r2max);
    if ((threadIdx.x & 31) == 0 && r2max) atomicMax(&rec.rmax2[b], r2max);
}

__global__ void prep_double_kernel(const __grid_constant__ BatchParams bp, const double *__restrict__ atoms,
                                   const void *__restrict__ amps, int amp_dtype, DoubleRecs rec) {
    const int b = blockIdx.y;
    const ImageDesc d = bp.img[b];
    const int64_t nrec = (int64_t)d.ntiles * bp.te;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nrec;
         j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = d.rec + j;
        if (j < d.n) {
            const int64_t s = d.src + j;
            rec.r64[r] = reinterpret_cast<const double4 *>(atoms)[s];
            double amp = 1.0;
            if (amps) amp = amp_dtype == IDIWF_F32 ? (double)static_cast<const float *>(amps)[s]
                                                  : static_cast<const double *>(amps)[s];
            rec.ra[r] = amp;
        } else {
            rec.r64[r] = make_double4(0, 0, 0, 0);
            rec.ra[r] = 0.0;
        }
    }
}

// ---------------------------------------------------------------------------
// output
// ---------------------------------------------------------------------------
__device__ __forceinline__ void store_pixel(void *out, int out_kind, int64_t idx, double re,
                                            double im) {
    switch (out_kind) {
        case IDIWF_OUT_C128:
            reinterpret_cast<double2 *>(out)[idx] = make_double2(re, im);
            break;
        case IDIWF_OUT_C64:
            reinterpret_cast<float2 *>(out)[idx] = make_float2((float)re, (float)im);
            break;
        case IDIWF_OUT_I64:
            reinterpret_cast<double *>(out)[idx] = re * re + im * im;
            break;
        default:
            reinterpret_cast<float *>(out)[idx] = (float)(re * re + im * im);
            break;
    }
}

// Final per-pixel step of the split forward: the far-field 1/|d| factor, the
// near-field constant phase k (|d| - d_z) (left out of the per-pair sum,
// applied here in FP64 for field outputs), then the store.
template <bool NF, bool SCALE>
__device__ __forceinline__ void finish_pixel(const GeomParams &g, int p, double re, double im, void *out,
                                             int out_kind, int64_t idx) {
    if ((!NF && SCALE) || (NF && out_kind <= IDIWF_OUT_C64)) {
        const int ix = p / g.ny, iy = p - ix * g.ny;
        double dx, dy, dz;
        pixel_cpu(g, ix, iy, dx, dy, dz);
        const double rho2 = dx * dx + dy * dy;
        const double D = sqrt(rho2 + dz * dz);
        if (!NF && SCALE) {
            re /= D;
            im /= D;
        }
        if (NF && out_kind <= IDIWF_OUT_C64) {
            const double c = g.kp * (dz > 0 ? rho2 / (D + dz) : D - dz);
            double sn, cs;
            sincospi(2.0 * (c - rint(c)), &sn, &cs);
            const double r2 = re * cs - im * sn;
            im = re * sn + im * cs;
            re = r2;
        }
    }
    store_pixel(out, out_kind, idx, re, im);
}

// Sum of the emitter-chunk partials of every pixel, in chunk order, then the
// final per-pixel step.  partials: [ksplit][n_images][npix] double2.
template <bool NF, bool SCALE>
__global__ void fwd_finish_kernel(const GeomParams g, const double2 *__restrict__ partials, int ksplit,
                                  int n_images, void *__restrict__ out, int out_kind) {
    const int npix = g.nx * g.ny;
    const int64_t total = (int64_t)n_images * npix;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        double re = 0.0, im = 0.0;
        for (int c = 0; c < ksplit; ++c) {
            const double2 v = partials[(int64_t)c * total + t];
            re += v.x;
            im += v.y;
        }
        finish_pixel<NF, SCALE>(g, (int)(t % npix), re, im, out, out_kind, t);
    }
}

// ---------------------------------------------------------------------------
// split-precision kernel
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// Constants of a run's base angle with the 8 low fixed-point bits, in units
// of pi_f = FP32 pi as in the per-pixel path: C is -pi_f (1.5 + 2^-8 + 2^-24)
// rounded to FP32 and S = pi_f 2^-8 minus C's rounding error, so that C + S
// is exact up to the FP32 rounding of S (< 5e-10 rad).
constexpr double kPiF = (double)3.14159274f;
constexpr double kRunBaseCExact = -kPiF * (1.5 + 1.0 / 256.0 + 1.0 / 16777216.0);
constexpr float kRunBaseC = (float)kRunBaseCExact;
constexpr float kRunBaseS = (float)(kPiF / 256.0 - ((double)kRunBaseC - kRunBaseCExact));

// Base point of run b of the thread whose first pixel is p0: the middle of
// the aligned run (rows hold a whole number of runs when runs are in use).
__device__ __forceinline__ PixelDir run_base(const GeomParams &g, int p0, int b, int npix) {
    const int rs = min((p0 & ~(kRun - 1)) + kRun * b, npix - kRun);
    const int ix = rs / g.ny;
    return pixel_dir(g, (double)ix, (double)(rs - ix * g.ny) + 0.5 * (kRun - 1));
}

// One work unit (image, pixel tile[, emitter chunk]) of the split kernel.
//
// PATH = kPathPixel: every pixel forms its phase with its own FP64 DFMA chain;
//   the near-field term h (|r|^2 - s^2), h = k / (2|d|), is added in FP32.
// PATH = kPathRuns: one FP64 chain per run of kRun pixels forms the phase at the
//   middle of the run (fixed point, half-turn fold as below); pixel i adds the
//   FP32 offset D_i . r with D_i = 2 pi (nq_i - nq_base) = -k (d_hat_i -
//   d_hat_base), exact up to FP32 rounding because |D_i . r| <= kGroupMaxPhase
//   (checked per image by the caller).  The near-field term uses
//   s_i = d_hat_i . r = s_base - D_i.r / k.  The half-turn sign of the base
//   applies to the whole run.
// PATH = kPathExact (near field only): as kPathPixel, but the quadratic term
//   k r_perp^2 / (2|d|) joins the FP64 chain (s = d_hat . r recovered from the
//   chain as z - (t - Psi)/kp, so r_perp^2 = |r|^2 - s^2 in FP64), and the
//   exact remainder R = h N (2s - N), N = r_perp^2 / (|d| + |d - r| - s), is
//   added in FP32 (|d - r| from a reciprocal square root, which also gives the
//   "scale" factor 1/|d - r|).
// Returns true when a bounded wait gave up (the unit is abandoned).
template <int PPT, bool NF, bool SCALE, bool SECOND, bool CHUNKED, int PATH>
__device__ __forceinline__ bool split_unit(const BatchParams &bp, const GeomParams &g, const SplitRecs &rec,
                                           void *__restrict__ out, int out_kind, WsHeader *__restrict__ hdr,
                                           double2 *__restrict__ partials, unsigned char *smem, uint64_t *bar,
                                           int *s_abort, uint32_t &issued, uint32_t &consumed, int img,
                                           int chunk, const ImageDesc &d, int p0, int tbeg, int tend,
                                           float *__restrict__ kahan) {
    constexpr bool GROUP = PATH == kPathRuns;
    constexpr bool EXACT = PATH == kPathExact;
    static_assert(!EXACT || NF, "the exact path is a near-field path");
    constexpr int PH = PPT / 2;
    constexpr int NB = PPT >= kRun ? PPT / kRun : 1;  // runs (base phases) per thread
    constexpr int NQ = GROUP ? NB : PPT;
    const int tid = threadIdx.x;
    const int TE = bp.te;
    const uint32_t stage_bytes = (uint32_t)TE * kSplitRecBytes;
    const int npix = g.nx * g.ny;
    const float2 PI2 = f2(3.14159274f, 3.14159274f);
    const float2 NEG_15PI2 = f2(-4.71238898f, -4.71238898f);

    // ---- per-pixel constants (FP64 geometry) ----
    // cx/cy/cz: d_hat of each pixel, or (GROUP) its offset coefficients D_i
    // (EXACT) hq: the quadratic term's FP64 coefficient kp / (2|d|) in turns,
    // dd: |d| in FP32
    double nqx[NQ], nqy[NQ], nqz[NQ], hq[EXACT ? PPT : 1];
    float2 cx[PH], cy[PH], cz[PH], hh[PH], iD[PH], iD2[PH], dd[EXACT ? PH : 1];
    float dbx[NB], dby[NB], dbz[NB];
    PixelDir base[NB];
    if (GROUP) {
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            base[b] = run_base(g, p0, b, npix);
            nqx[b] = base[b].nqx;
            nqy[b] = base[b].nqy;
            nqz[b] = base[b].nqz;
            dbx[b] = (float)base[b].ux;
            dby[b] = (float)base[b].uy;
            dbz[b] = (float)base[b].uz;
        }
    }
#pragma unroll
    for (int i = 0; i < PPT; ++i) {
        const int p = min(p0 + i, npix - 1);
        const int ix = p / g.ny, iy = p - ix * g.ny;
        const PixelDir q = pixel_dir(g, (double)ix, (double)iy);
        float fx, fy, fz;
        if (GROUP) {
            const PixelDir &bs = base[PPT >= kRun ? i / kRun : 0];
            fx = (float)(kTwoPi * (q.nqx - bs.nqx));
            fy = (float)(kTwoPi * (q.nqy - bs.nqy));
            fz = (float)(kTwoPi * (q.nqz - bs.nqz));
        } else {
            nqx[i] = q.nqx;
            nqy[i] = q.nqy;
            nqz[i] = q.nqz;
            fx = (float)q.ux;
            fy = (float)q.uy;
            fz = (float)q.uz;
        }
        const float fh = (float)(-g.k * 0.5 * q.invD);  // -h, pairs with the negated w
        const float fi = (float)q.invD, fi2 = (float)(q.invD * q.invD);
        float fd = 0.f;
        if (EXACT) {
            hq[i] = 0.5 * g.kp * q.invD;
            fd = (float)(1.0 / q.invD);
        }
        if (i & 1) {
            cx[i / 2].y = fx; cy[i / 2].y = fy; cz[i / 2].y = fz;
            hh[i / 2].y = fh; iD[i / 2].y = fi; iD2[i / 2].y = fi2;
            if (EXACT) dd[i / 2].y = fd;
        } else {
            cx[i / 2].x = fx; cy[i / 2].x = fy; cz[i / 2].x = fz;
            hh[i / 2].x = fh; iD[i / 2].x = fi; iD2[i / 2].x = fi2;
            if (EXACT) dd[i / 2].x = fd;
        }
    }
    const float ninvk = (float)(-1.0 / g.k);
    const float2 NEG_INVK2 = f2(ninvk, ninvk);

    // Kahan-compensated totals per pixel (sum, compensation; re, im).  The run
    // kernel keeps them in shared memory, [4 PPT][threads] (touched once per
    // kFold emitters), to leave its registers to the emitter loop.
    float sre[GROUP ? 1 : PPT], cre[GROUP ? 1 : PPT], sim[GROUP ? 1 : PPT], cim[GROUP ? 1 : PPT];
    const int nthr = blockDim.x;
#pragma unroll
    for (int i = 0; i < PPT; ++i) {
        if (GROUP) {
#pragma unroll
            for (int c = 0; c < 4; ++c) kahan[(c * PPT + i) * nthr + tid] = 0.0f;
        } else {
            sre[i] = cre[i] = sim[i] = cim[i] = 0.0f;
        }
    }

    const int nt = tend - tbeg;
    if (tid == 0) {
        for (int s = 0; s < 2 && s < nt; ++s) {
            const uint32_t slot = issued & 1;
            unsigned char *st = smem + slot * stage_bytes;
            const int64_t r0 = d.rec + (int64_t)(tbeg + s) * TE;
            mbar_arrive_expect_tx(&bar[slot], stage_bytes);
            bulk_g2s(st, rec.r64 + r0, TE * 32, &bar[slot]);
            bulk_g2s(st + TE * 32, rec.rA + r0, TE * 16, &bar[slot]);
            bulk_g2s(st + TE * 48, rec.rC + r0, TE * 4, &bar[slot]);
            ++issued;
        }
    }
    for (int it = 0; it < nt; ++it) {
        const uint32_t slot = consumed & 1;
        if (!mbar_wait_bounded(&bar[slot], (consumed >> 1) & 1)) {
            record_error(&hdr->error, kErrTimeout);
            *s_abort = 1;
        }
        const unsigned char *st = smem + slot * stage_bytes;
        const double4 *s64 = reinterpret_cast<const double4 *>(st);
        const float4 *sA = reinterpret_cast<const float4 *>(st + TE * 32);
        const float *sC = reinterpret_cast<const float *>(st + TE * 48);

        for (int jb = 0; jb < TE; jb += kFold) {
            float2 are[PH], aim[PH];
#pragma unroll
            for (int q = 0; q < PH; ++q) are[q] = aim[q] = f2(0.f, 0.f);
            if (GROUP) {
#pragma unroll(PPT <= 4 ? 4 : 2)
                for (int j = jb; j < jb + kFold; ++j) {
                    const double4 r = s64[j];
                    const float4 A = sA[j];
                    const float a1 = sC[j];
                    const float2 X2 = f2(A.x, A.x), Y2 = f2(A.y, A.y), Z2 = f2(A.z, A.z);
                    float2 XB2[NB], AS2[NB], SB2[NB];
#pragma unroll
                    for (int b = 0; b < NB; ++b) {
                        double t = __fma_rn(nqx[b], r.x, r.w);
                        t = __fma_rn(nqy[b], r.y, t);
                        t = __fma_rn(nqz[b], r.z, t);
                        const uint32_t lo = (uint32_t)__double2loint(t);
                        // base angle and half-turn sign as in the per-pixel path below,
                        // plus the 8 fixed-point bits below the 23 kept there:
                        // pi u + C + (1 + r 2^-23) S = pi (u - 1.5) + pi r 2^-31 - pi 2^-24
                        // (the last term takes back the record's half-step rounding offset)
                        float xb = __fmaf_rn(__uint_as_float(((lo >> 8) & 0x007FFFFFu) | 0x3F800000u),
                                             PI2.x, kRunBaseC);
                        xb = __fmaf_rn(__uint_as_float((lo & 0xFFu) | 0x3F800000u), kRunBaseS, xb);
                        const float as = __uint_as_float(__float_as_uint(a1) ^ (lo & 0x80000000u));
                        XB2[b] = f2(xb, xb);
                        AS2[b] = f2(as, as);
                        SB2[b] = f2(0.f, 0.f);
                        if (NF) {
                            const float sb = __fmaf_rn(dbz[b], A.z, __fmaf_rn(dby[b], A.y, __fmul_rn(dbx[b], A.x)));
                            SB2[b] = f2(sb, sb);
                        }
                    }
#pragma unroll
                    for (int q = 0; q < PH; ++q) {
                        const int b = PPT >= kRun ? q / (kRun / 2) : 0;
                        float2 dl = __fmul2_rn(cx[q], X2);
                        dl = __ffma2_rn(cy[q], Y2, dl);
                        dl = __ffma2_rn(cz[q], Z2, dl);
                        float2 amp = AS2[b];
                        if (NF) {
                            const float2 s = __ffma2_rn(dl, NEG_INVK2, SB2[b]);
                            const float2 w2 = __ffma2_rn(s, s, f2(A.w, A.w));
                            dl = __ffma2_rn(hh[q], w2, dl);
                            if (SCALE) amp = __fmul2_rn(AS2[b], __ffma2_rn(s, iD2[q], iD[q]));
                        } else if (SECOND) {
                            dl = __ffma2_rn(hh[q], f2(A.w, A.w), dl);  // (-h)(-(x^2+y^2))
                        }
                        const float2 arg = __fadd2_rn(XB2[b], dl);
                        float s0, c0, s1, c1;
                        __sincosf(arg.x, &s0, &c0);
                        __sincosf(arg.y, &s1, &c1);
                        are[q] = __ffma2_rn(amp, f2(c0, c1), are[q]);
                        aim[q] = __ffma2_rn(amp, f2(s0, s1), aim[q]);
                    }
                }
            } else {
#pragma unroll(PPT <= 4 ? 4 : 2)
                for (int j = jb; j < jb + kFold; ++j) {
                    const double4 r = s64[j];
                    const float4 A = sA[j];
                    const float a1 = sC[j];
                    const float2 a2 = f2(a1, a1);
                    double rr = 0.0;  // (EXACT) |r|^2 in FP64
                    if (EXACT) rr = __fma_rn(r.z, r.z, __fma_rn(r.y, r.y, r.x * r.x));
#pragma unroll
                    for (int q = 0; q < PH; ++q) {
                        uint32_t lo[2];
#pragma unroll
                        for (int e = 0; e < 2; ++e) {
                            const int i = 2 * q + e;
                            double t = __fma_rn(nqx[i], r.x, r.w);
                            t = __fma_rn(nqy[i], r.y, t);
                            t = __fma_rn(nqz[i], r.z, t);
                            if (EXACT) {
                                // t - Psi = nq . r = kp (z - s) exactly (same binade)
                                const double sd = __fma_rn(-g.ikp, t - r.w, r.z);
                                t = __fma_rn(hq[i], __fma_rn(-sd, sd, rr), t);
                            }
                            lo[e] = (uint32_t)__double2loint(t);
                        }
                        // phase = n*pi + x, x = pi*(u - 1.5) in [-pi/2, pi/2): u from
                        // bits 30..8; odd n (bit 31) negates the term, folded into
                        // the amplitude's sign.  Mapping both halves of the circle
                        // onto one half and flipping the sign makes the mean error
                        // of the hardware cosine cancel over the circle instead of
                        // adding up coherently over emitters.
                        const float2 u = f2(__uint_as_float(((lo[0] >> 8) & 0x007FFFFFu) | 0x3F800000u),
                                            __uint_as_float(((lo[1] >> 8) & 0x007FFFFFu) | 0x3F800000u));
                        float2 arg = __ffma2_rn(u, PI2, NEG_15PI2);
                        float2 amp = a2;
                        if (NF) {
                            float2 s = __fmul2_rn(cx[q], f2(A.x, A.x));
                            s = __ffma2_rn(cy[q], f2(A.y, A.y), s);
                            s = __ffma2_rn(cz[q], f2(A.z, A.z), s);
                            const float2 w2 = __ffma2_rn(s, s, f2(A.w, A.w));  // s^2 - |r|^2
                            if (EXACT) {
                                // L^2 = |d|(|d| - 2s) + |r|^2, N = r_perp^2 / (|d| + L - s),
                                // R = h N (2s - N) = (-h)(-N)(2s - N)
                                const float2 l2 = __ffma2_rn(__ffma2_rn(s, f2(-2.f, -2.f), dd[q]), dd[q],
                                                             f2(-A.w, -A.w));
                                const float2 y = f2(rsqrt_approx(l2.x), rsqrt_approx(l2.y));
                                const float2 den = __ffma2_rn(s, f2(-1.f, -1.f), __ffma2_rn(l2, y, dd[q]));
                                const float2 nN = __fmul2_rn(w2, f2(rcp_approx(den.x), rcp_approx(den.y)));
                                arg = __ffma2_rn(__fmul2_rn(hh[q], nN), __ffma2_rn(s, f2(2.f, 2.f), nN), arg);
                                if (SCALE) amp = __fmul2_rn(a2, y);
                            } else {
                                // -h (s^2 - |r|^2) = h (|r|^2 - s^2)
                                arg = __ffma2_rn(hh[q], w2, arg);
                                if (SCALE) amp = __fmul2_rn(a2, __ffma2_rn(s, iD2[q], iD[q]));
                            }
                        } else if (SECOND) {
                            arg = __ffma2_rn(hh[q], f2(A.w, A.w), arg);  // (-h)(-(x^2+y^2))
                        }
                        amp.x = __uint_as_float(__float_as_uint(amp.x) ^ (lo[0] & 0x80000000u));
                        amp.y = __uint_as_float(__float_as_uint(amp.y) ^ (lo[1] & 0x80000000u));
                        float s0, c0, s1, c1;
                        __sincosf(arg.x, &s0, &c0);
                        __sincosf(arg.y, &s1, &c1);
                        are[q] = __ffma2_rn(amp, f2(c0, c1), are[q]);
                        aim[q] = __ffma2_rn(amp, f2(s0, s1), aim[q]);
                    }
                }
            }
            // Kahan fold of the block partials
#pragma unroll
            for (int q = 0; q < PH; ++q) {
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int i = 2 * q + e;
                    const float pr = e ? are[q].y : are[q].x;
                    const float pi = e ? aim[q].y : aim[q].x;
                    if (GROUP) {
                        float *k0 = kahan + (0 * PPT + i) * nthr + tid, *k1 = kahan + (1 * PPT + i) * nthr + tid;
                        float *k2 = kahan + (2 * PPT + i) * nthr + tid, *k3 = kahan + (3 * PPT + i) * nthr + tid;
                        const float s0 = *k0, c0 = *k1, s1 = *k2, c1 = *k3;
                        float y = pr - c0;
                        float t = s0 + y;
                        *k1 = (t - s0) - y;
                        *k0 = t;
                        y = pi - c1;
                        t = s1 + y;
                        *k3 = (t - s1) - y;
                        *k2 = t;
                    } else {
                        float y = pr - cre[i];
                        float t = sre[i] + y;
                        cre[i] = (t - sre[i]) - y;
                        sre[i] = t;
                        y = pi - cim[i];
                        t = sim[i] + y;
                        cim[i] = (t - sim[i]) - y;
                        sim[i] = t;
                    }
                }
            }
        }
        ++consumed;
        __syncthreads();
        if (*s_abort) return true;
        if (tid == 0 && it + 2 < nt) {
            const uint32_t slot2 = issued & 1;
            unsigned char *st2 = smem + slot2 * stage_bytes;
            const int64_t r0 = d.rec + (int64_t)(tbeg + it + 2) * TE;
            mbar_arrive_expect_tx(&bar[slot2], stage_bytes);
            bulk_g2s(st2, rec.r64 + r0, TE * 32, &bar[slot2]);
            bulk_g2s(st2 + TE * 32, rec.rA + r0, TE * 16, &bar[slot2]);
            bulk_g2s(st2 + TE * 48, rec.rC + r0, TE * 4, &bar[slot2]);
            ++issued;
        }
    }

    const int64_t obase = (int64_t)img * npix;
#pragma unroll
    for (int i = 0; i < PPT; ++i) {
        const int p = p0 + i;
        if (p < npix) {
            double re, im;
            if (GROUP) {
                re = (double)kahan[(0 * PPT + i) * nthr + tid] - (double)kahan[(1 * PPT + i) * nthr + tid];
                im = (double)kahan[(2 * PPT + i) * nthr + tid] - (double)kahan[(3 * PPT + i) * nthr + tid];
            } else {
                re = (double)sre[i] - (double)cre[i];
                im = (double)sim[i] - (double)cim[i];
            }
            if (CHUNKED)
                partials[((int64_t)chunk * bp.n_images + img) * npix + p] = make_double2(re, im);
            else
                finish_pixel<NF, SCALE>(g, p, re, im, out, out_kind, obase + p);
        }
    }
    return false;
}

// The split forward is up to three kernels launched back to back, one per
// path (split_path: pixel runs, per-pixel FP64 phase, exact near field), each
// taking the units of its own images from its own work counter.  Without the
// per-pixel path's registers the run kernel fits three 256-thread CTAs per SM
// (two for the others).  A kernel whose path no image of the launch takes
// returns at once.  The per-pixel kernel, which every launch runs, reports
// images outside the split kernels' range (kErrGeometry); no kernel takes them.
// Every CTA classifies the images once, into shared memory: a square root or
// the classifier's arithmetic in the persistent loop costs the run kernel
// several percent of its speed.
template <int PPT, bool NF, bool SCALE, bool SECOND, bool CHUNKED, int PATH>
__global__ void __launch_bounds__(256, (PPT <= 4 ? (PATH == kPathRuns ? 3 : 2) : 1))
    fwd_split_kernel(const __grid_constant__ BatchParams bp, const GeomParams g, SplitRecs rec,
                     void *__restrict__ out, int out_kind, WsHeader *__restrict__ hdr,
                     uint64_t *__restrict__ cta_ns, double2 *__restrict__ partials) {
    static_assert(PPT % 2 == 0, "pixels are processed in f32x2 pairs");
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int s_unit, s_abort;
    __shared__ uint8_t s_path[kMaxImagesPerLaunch];

    const int tid = threadIdx.x;
    bool mine = false;
    for (int i = tid; i < bp.n_images; i += blockDim.x) {
        const int path = split_path(g, rec.rmax2[i], bp.groups != 0, false);
        s_path[i] = (uint8_t)path;
        mine |= path == PATH;
        if (PATH == kPathPixel && path == kPathReject && blockIdx.x == 0) record_error(&hdr->error, kErrGeometry);
    }
    if (!__syncthreads_or(mine)) return;
    uint32_t *counter = PATH == kPathRuns ? &hdr->work_counter
                                          : (PATH == kPathPixel ? &hdr->work_counter2 : &hdr->work_counter3);

    const uint64_t t_start = globaltimer_ns();
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        s_abort = 0;
        mbar_fence_init();
        if (blockIdx.x == 0) hdr->n_ctas = gridDim.x;
    }
    __syncthreads();

    const int tile_px = blockDim.x * PPT;
    uint32_t issued = 0, consumed = 0;
    bool aborted = false;

    const int ks = CHUNKED ? bp.ksplit : 1;
    for (;;) {
        __syncthreads();
        if (tid == 0) {
            // next unit of this kernel's path (units of the other kernel are
            // skipped here, out of the CTA's control flow)
            int u;
            for (;;) {
                u = (int)atomicAdd(counter, 1u);
                if (u >= bp.total_units || s_path[bp.order[u / ks / bp.tiles_per_image]] == PATH) break;
            }
            s_unit = u;
        }
        __syncthreads();
        const int unit = s_unit;
        if (unit >= bp.total_units) break;
        const int chunk = unit % ks;
        const int pu = unit / ks;
        const int img = bp.order[pu / bp.tiles_per_image];
        const int ptile = pu % bp.tiles_per_image;
        const ImageDesc d = bp.img[img];
        const int p0 = ptile * tile_px + tid * PPT;
        // emitter tiles of this unit: the whole image, or one chunk of it
        const int tbeg = CHUNKED ? min(chunk * d.tpc, d.ntiles) : 0;
        const int tend = CHUNKED ? min(tbeg + d.tpc, d.ntiles) : d.ntiles;
        if (split_unit<PPT, NF, SCALE, SECOND, CHUNKED, PATH>(
                bp, g, rec, out, out_kind, hdr, partials, smem, bar, &s_abort, issued, consumed, img, chunk, d, p0,
                tbeg, tend, reinterpret_cast<float *>(smem + 2 * (size_t)bp.te * kSplitRecBytes))) {
            aborted = true;
            break;
        }
    }
    if (aborted) {
        // wait (bounded) for copies still in flight into this CTA's shared memory
        if (tid == 0)
            while (consumed < issued) {
                mbar_wait_bounded(&bar[consumed & 1], (consumed >> 1) & 1);
                ++consumed;
            }
        return;
    }
    if (tid == 0) cta_ns[blockIdx.x] = globaltimer_ns() - t_start;
}

// ---------------------------------------------------------------------------
// all-FP64 kernel (reference rounding sequence)
// ---------------------------------------------------------------------------
template <int PPT, bool NF, bool SCALE, bool SECOND, bool ACC = false>
__global__ void __launch_bounds__(256) fwd_double_kernel(const __grid_constant__ BatchParams bp,
                                                         const GeomParams g, DoubleRecs rec,
                                                         void *__restrict__ out, int out_kind,
                                                         WsHeader *__restrict__ hdr,
                                                         uint64_t *__restrict__ cta_ns) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int s_unit, s_abort;

    const int tid = threadIdx.x;
    const int TE = bp.te;
    const uint32_t stage_bytes = (uint32_t)TE * kDoubleRecBytes;
    const uint64_t t_start = globaltimer_ns();
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        s_abort = 0;
        mbar_fence_init();
        if (blockIdx.x == 0) hdr->n_ctas = gridDim.x;
    }
    __syncthreads();
    const int npix = g.nx * g.ny;
    const int tile_px = blockDim.x * PPT;
    uint32_t issued = 0, consumed = 0;
    bool aborted = false;

    for (;;) {
        __syncthreads();
        if (tid == 0) s_unit = (int)atomicAdd(&hdr->work_counter, 1u);
        __syncthreads();
        const int unit = s_unit;
        if (unit >= bp.total_units) break;
        const int img = bp.order[unit / bp.tiles_per_image];
        const int ptile = unit % bp.tiles_per_image;
        const ImageDesc d = bp.img[img];
        const int p0 = ptile * tile_px + tid * PPT;

        double px[PPT], py[PPT], pz[PPT], qx[PPT], qy[PPT], qz[PPT], rdist[PPT], c2[PPT];
#pragma unroll
        for (int i = 0; i < PPT; ++i) {
            const int p = min(p0 + i, npix - 1);
            const int ix = p / g.ny, iy = p - ix * g.ny;
            pixel_cpu(g, ix, iy, px[i], py[i], pz[i]);
            // cpu.py:86-89
            rdist[i] = __drcp_rn(__dsqrt_rn(
                __dadd_rn(__dadd_rn(__dmul_rn(px[i], px[i]), __dmul_rn(py[i], py[i])), __dmul_rn(pz[i], pz[i]))));
            qz[i] = __dmul_rn(g.k, __dsub_rn(__dmul_rn(pz[i], rdist[i]), 1.0));
            qx[i] = __dmul_rn(g.k, __dmul_rn(px[i], rdist[i]));
            qy[i] = __dmul_rn(g.k, __dmul_rn(py[i], rdist[i]));
            c2[i] = __dmul_rn(g.k, rdist[i]) * 0.5;
            if (ACC) {
                // accurate near field: the pixel constant k (|d| - d_z) in
                // turns, without cancellation (reuses the far-field slots)
                const double rho2 = px[i] * px[i] + py[i] * py[i];
                const double D = sqrt(rho2 + pz[i] * pz[i]);
                const double cc = g.kp * (pz[i] > 0 ? rho2 / (D + pz[i]) : D - pz[i]);
                qx[i] = D;
                qy[i] = cc - rint(cc);
            }
        }
        double ax[PPT], ay[PPT], cx[PPT], cy[PPT];
#pragma unroll
        for (int i = 0; i < PPT; ++i) ax[i] = ay[i] = cx[i] = cy[i] = 0.0;

        const int nt = d.ntiles;
        if (tid == 0) {
            for (int s = 0; s < 2 && s < nt; ++s) {
                const uint32_t slot = issued & 1;
                unsigned char *st = smem + slot * stage_bytes;
                const int64_t r0 = d.rec + (int64_t)s * TE;
                mbar_arrive_expect_tx(&bar[slot], stage_bytes);
                bulk_g2s(st, rec.r64 + r0, TE * 32, &bar[slot]);
                bulk_g2s(st + TE * 32, rec.ra + r0, TE * 8, &bar[slot]);
                ++issued;
            }
        }
        for (int it = 0; it < nt; ++it) {
            const uint32_t slot = consumed & 1;
            if (!mbar_wait_bounded(&bar[slot], (consumed >> 1) & 1)) {
                record_error(&hdr->error, kErrTimeout);
                s_abort = 1;
            }
            const unsigned char *st = smem + slot * stage_bytes;
            const double4 *s64 = reinterpret_cast<const double4 *>(st);
            const double *sa = reinterpret_cast<const double *>(st + TE * 32);
            const int jend = min(TE, d.n - it * TE);
            for (int j = 0; j < jend; ++j) {
                const double4 r = s64[j];
                const double aj = sa[j];
#pragma unroll
                for (int i = 0; i < PPT; ++i) {
                    double phase, w = 1.0;
                    if (NF) {
                        // cpu.py:44-47 with numba's contraction
                        const double a = __dsub_rn(px[i], r.x), b = __dsub_rn(py[i], r.y),
                                     c = __dsub_rn(pz[i], r.z);
                        const double dist = __dsqrt_rn(__fma_rn(c, c, __fma_rn(a, a, __dmul_rn(b, b))));
                        if (ACC) {
                            // |d-r| - |d| = (|r|^2 - 2 d.r) / (|d-r| + |d|): no cancellation
                            const double rr = fma(r.z, r.z, fma(r.x, r.x, r.y * r.y));
                            const double dr = fma(pz[i], r.z, fma(px[i], r.x, py[i] * r.y));
                            const double delta = (rr - 2.0 * dr) / (dist + qx[i]);
                            phase = fma(kTwoPi, qy[i], fma(g.k, delta + r.z, r.w));
                        } else {
                            phase = __fma_rn(__dadd_rn(__dsub_rn(dist, pz[i]), r.z), g.k, r.w);
                        }
                        if (SCALE) w = __drcp_rn(dist);
                    } else {
                        // cpu.py:59
                        phase = __dadd_rn(-__fma_rn(r.z, qz[i], __fma_rn(r.x, qx[i], __dmul_rn(r.y, qy[i]))), r.w);
                        if (SECOND)  // sim.cu:88
                            phase = __dadd_rn(phase, __dmul_rn(c2[i], __dadd_rn(__dmul_rn(r.x, r.x), __dmul_rn(r.y, r.y))));
                        if (SCALE) w = rdist[i];
                    }
                    w = __dmul_rn(w, aj);
                    double sn, cs;
                    sincos(phase, &sn, &cs);
                    const double vx = __dmul_rn(w, cs), vy = __dmul_rn(w, sn);
                    // Kahan, cpu.py:97-105
                    const double yx = __dsub_rn(vx, cx[i]), yy = __dsub_rn(vy, cy[i]);
                    const double tx = __dadd_rn(ax[i], yx), ty = __dadd_rn(ay[i], yy);
                    cx[i] = __dsub_rn(__dsub_rn(tx, ax[i]), yx);
                    cy[i] = __dsub_rn(__dsub_rn(ty, ay[i]), yy);
                    ax[i] = tx;
                    ay[i] = ty;
                }
            }
            ++consumed;
            __syncthreads();
            if (s_abort) {
                aborted = true;
                break;
            }
            if (tid == 0 && it + 2 < nt) {
                const uint32_t slot2 = issued & 1;
                unsigned char *st2 = smem + slot2 * stage_bytes;
                const int64_t r0 = d.rec + (int64_t)(it + 2) * TE;
                mbar_arrive_expect_tx(&bar[slot2], stage_bytes);
                bulk_g2s(st2, rec.r64 + r0, TE * 32, &bar[slot2]);
                bulk_g2s(st2 + TE * 32, rec.ra + r0, TE * 8, &bar[slot2]);
                ++issued;
            }
        }
        if (aborted) break;
        const int64_t obase = (int64_t)img * npix;
#pragma unroll
        for (int i = 0; i < PPT; ++i) {
            const int p = p0 + i;
            if (p < npix) store_pixel(out, out_kind, obase + p, ax[i], ay[i]);
        }
    }
    if (aborted) {
        if (tid == 0)
            while (consumed < issued) {
                mbar_wait_bounded(&bar[consumed & 1], (consumed >> 1) & 1);
                ++consumed;
            }
        return;
    }
    if (tid == 0) cta_ns[blockIdx.x] = globaltimer_ns() - t_start;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

struct LaunchShape {
    int threads, ppt, te, ctas_per_sm;
    int groups = 1;  // split: pixel runs with a base phase where bounded
};

static int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (!cached[dev]) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cached[dev] = n > 0 ? n : 148;
    }
    return cached[dev];
}

GeomParams make_geom(const idiwf_geom *g) {
    GeomParams p;
    p.nx = g->nx;
    p.ny = g->ny;
    p.flags = g->flags;
    p.has_rot = g->has_rot;
    p.pixelsize = g->pixelsize;
    p.detz = g->detz;
    p.k = g->k;
    p.kp = g->k * kInvTwoPi;
    p.ikp = kTwoPi / g->k;
    p.offx = g->offset[0];
    p.offy = g->offset[1];
    for (int i = 0; i < 9; ++i) p.rot[i] = g->has_rot ? g->rot[i] : (i % 4 == 0 ? 1.0 : 0.0);
    // pixel (px, py) sits at px c0 + py c1 + detz c2 (columns of rot); rows run along c1
    const double *M = p.rot;
    const double c0[3] = {M[0], M[3], M[6]}, c1[3] = {M[1], M[4], M[7]}, c2[3] = {M[2], M[5], M[8]};
    const double n[3] = {c0[1] * c1[2] - c0[2] * c1[1], c0[2] * c1[0] - c0[0] * c1[2], c0[0] * c1[1] - c0[1] * c1[0]};
    const double nn = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    const double h = nn > 0 ? std::fabs(g->detz * (c2[0] * n[0] + c2[1] * n[1] + c2[2] * n[2])) / nn : 0.0;
    const double half = 0.5 * (kRun - 1) * std::fabs(g->pixelsize) * std::sqrt(c1[0] * c1[0] + c1[1] * c1[1] + c1[2] * c1[2]);
    p.run_span = h > 0 ? half / h : INFINITY;
    p.dmin = h;
    p.inv_dmin2 = h > 0 ? 1.0 / (h * h) : INFINITY;
    const double c3 = h > 0 ? kNfBoundC * g->k / (h * h) : INFINITY;
    p.nf_c3 = c3 * c3;
    return p;
}

static idiwf_status validate_geom(const idiwf_geom *g) {
    if (!g) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "geom is NULL");
    if (g->nx <= 0 || g->ny <= 0)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "detector size must be positive");
    if ((int64_t)g->nx * g->ny >= (int64_t)1 << 31)
        return set_error(IDIWF_ERR_UNSUPPORTED, "detector has 2^31 or more pixels");
    if (!(g->k > 0) || !std::isfinite(g->k))
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "k must be positive and finite");
    if (!std::isfinite(g->pixelsize) || !std::isfinite(g->detz))
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "pixelsize/detz must be finite");
    if (g->flags & ~(IDIWF_NF | IDIWF_SCALE | IDIWF_SECONDORDER | IDIWF_ACCURATE))
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "unknown geometry flag");
    return IDIWF_OK;
}

static idiwf_status validate_batch(const idiwf_batch *b) {
    if (!b) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "batch is NULL");
    if (b->n_images <= 0) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "batch has no images");
    if (!b->offsets) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "batch offsets are NULL");
    if (b->offsets[0] != 0) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "offsets[0] must be 0");
    for (int i = 0; i < b->n_images; ++i) {
        const int64_t n = b->offsets[i + 1] - b->offsets[i];
        if (n < 0) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "offsets must be non-decreasing");
        if (n >= ((int64_t)1 << 30)) return set_error(IDIWF_ERR_UNSUPPORTED, "image with 2^30 or more emitters");
    }
    if (b->offsets[b->n_images] > 0 && !b->atoms)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "atoms pointer is NULL");
    if (b->atoms && (reinterpret_cast<uintptr_t>(b->atoms) & 31))
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "atoms must be 32-byte aligned");
    if (b->amplitudes && b->amp_dtype != IDIWF_F64 && b->amp_dtype != IDIWF_F32)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "amp_dtype must be IDIWF_F64 or IDIWF_F32");
    return IDIWF_OK;
}

// --- tuned shape cache ------------------------------------------------------
struct TuneKey {
    int precision, flags, nx, ny, nbucket;
    bool operator<(const TuneKey &o) const {
        return std::tie(precision, flags, nx, ny, nbucket) < std::tie(o.precision, o.flags, o.nx, o.ny, o.nbucket);
    }
};
static std::mutex g_tune_mu;
static std::map<TuneKey, LaunchShape> g_tune_cache;

static int n_bucket(const idiwf_batch *b) {
    const double mean = (double)b->offsets[b->n_images] / b->n_images;
    return mean <= 0 ? 0 : (int)std::floor(std::log2(mean));
}

static LaunchShape default_shape(int precision) {
    if (precision == IDIWF_SPLIT) return LaunchShape{256, 4, 512, 3};
    return LaunchShape{128, 2, 128, 2};
}

static idiwf_status resolve_shape(const idiwf_geom *g, const idiwf_batch *b, int precision,
                                  const idiwf_config *cfg, LaunchShape &s) {
    s = default_shape(precision);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(TuneKey{precision, g->flags, g->nx, g->ny, n_bucket(b)});
        if (it != g_tune_cache.end()) s = it->second;
    }
    if (cfg) {
        if (cfg->threads) s.threads = cfg->threads;
        if (cfg->pixels_per_thread) s.ppt = cfg->pixels_per_thread;
        if (cfg->emitters_per_tile) s.te = cfg->emitters_per_tile;
        if (cfg->ctas_per_sm) s.ctas_per_sm = cfg->ctas_per_sm;
        if (cfg->pixel_groups) s.groups = cfg->pixel_groups > 0;
    }
    if (s.threads != 64 && s.threads != 128 && s.threads != 256)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "threads must be 64, 128 or 256");
    if (precision == IDIWF_SPLIT) {
        if (s.ppt != 2 && s.ppt != 4 && s.ppt != 8)
            return set_error(IDIWF_ERR_INVALID_ARGUMENT, "split pixels_per_thread must be 2, 4 or 8");
        if (s.te < kFold || s.te > kChunkEmitters || (s.te & (s.te - 1)))
            return set_error(IDIWF_ERR_INVALID_ARGUMENT, "split emitters_per_tile must be a power of two in [64,1024]");
    } else {
        if (s.ppt != 1 && s.ppt != 2 && s.ppt != 4)
            return set_error(IDIWF_ERR_INVALID_ARGUMENT, "double pixels_per_thread must be 1, 2 or 4");
        if (s.te < 16 || s.te > 1024 || s.te % 16)
            return set_error(IDIWF_ERR_INVALID_ARGUMENT, "double emitters_per_tile must be a multiple of 16 in [16,1024]");
    }
    if (s.ctas_per_sm < 1 || s.ctas_per_sm > 8)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "ctas_per_sm must be in [1,8]");
    return IDIWF_OK;
}

static int64_t total_records(const idiwf_batch *b, int te) {
    int64_t t = 0;
    for (int i = 0; i < b->n_images; ++i) {
        const int64_t n = b->offsets[i + 1] - b->offsets[i];
        t += (n + te - 1) / te * te;
    }
    return t;
}

// Emitter chunks per (image, pixel tile) for the split kernel: 1 when the
// batch has pixel tiles for at least 3/4 of one wave of CTA slots (two per
// SM), else about two waves' worth of units.  Depends only on the problem and
// the SM count (not on the kernel shape), so the summation order is the same
// for every shape.
static int choose_ksplit(const idiwf_geom *g, const idiwf_batch *b) {
    const int npix = g->nx * g->ny;
    const int64_t base = (int64_t)std::min(b->n_images, kMaxImagesPerLaunch) * ((npix + 1023) / 1024);
    const int64_t slots = 2 * (int64_t)sm_count();
    if (4 * base >= 3 * slots) return 1;
    int64_t nmax = 0;
    for (int i = 0; i < b->n_images; ++i) nmax = std::max<int64_t>(nmax, b->offsets[i + 1] - b->offsets[i]);
    int64_t k = (2 * slots + base / 2) / base;
    k = std::min<int64_t>(k, (nmax + kChunkEmitters - 1) / kChunkEmitters);
    return (int)std::max<int64_t>(1, std::min<int64_t>(k, 64));
}

static size_t partials_bytes(const idiwf_geom *g, const idiwf_batch *b, int ksplit) {
    if (ksplit <= 1) return 0;
    return align256((size_t)ksplit * std::min(b->n_images, kMaxImagesPerLaunch) * g->nx * g->ny * 16);
}

static size_t forward_ws_bytes(const idiwf_geom *g, const idiwf_batch *b, int precision, const LaunchShape &s) {
    const int64_t nrec = std::max<int64_t>(total_records(b, s.te), 1);
    if (precision != IDIWF_SPLIT) return kWsDataOffset + double_recs_bytes(nrec);
    return kWsDataOffset + split_recs_bytes(nrec) + partials_bytes(g, b, choose_ksplit(g, b));
}

// Dynamic shared memory of a forward kernel: two stages of emitter records,
// plus for the pixel-run kernel the Kahan totals (4 floats per pixel of the CTA).
static size_t fwd_smem(int precision, const LaunchShape &s, int path) {
    if (precision != IDIWF_SPLIT) return 2 * (size_t)s.te * kDoubleRecBytes;
    return 2 * (size_t)s.te * kSplitRecBytes + (path == kPathRuns ? (size_t)16 * s.ppt * s.threads : 0);
}

// kernel table ---------------------------------------------------------------
template <int PPT, bool CH, int PATH>
static void *split_kernel_for3(int flags) {
    const bool nf = flags & IDIWF_NF, sc = flags & IDIWF_SCALE, so = flags & IDIWF_SECONDORDER;
    if (nf) return sc ? (void *)fwd_split_kernel<PPT, true, true, false, CH, PATH>
                      : (void *)fwd_split_kernel<PPT, true, false, false, CH, PATH>;
    if (PATH == kPathExact) return nullptr;  // near field only
    constexpr int P = PATH == kPathExact ? kPathPixel : PATH;
    if (so) return sc ? (void *)fwd_split_kernel<PPT, false, true, true, CH, P>
                      : (void *)fwd_split_kernel<PPT, false, false, true, CH, P>;
    return sc ? (void *)fwd_split_kernel<PPT, false, true, false, CH, P>
              : (void *)fwd_split_kernel<PPT, false, false, false, CH, P>;
}
// path: kPathRuns, kPathPixel or kPathExact (nullptr for the exact path
// without "nf")
template <int PPT, bool CH>
static void *split_kernel_for2(int flags, int path) {
    if (path == kPathRuns) return split_kernel_for3<PPT, CH, kPathRuns>(flags);
    if (path == kPathExact) return split_kernel_for3<PPT, CH, kPathExact>(flags);
    return split_kernel_for3<PPT, CH, kPathPixel>(flags);
}
template <int PPT>
static void *split_kernel_for(int flags, bool chunked, int path) {
    return chunked ? split_kernel_for2<PPT, true>(flags, path) : split_kernel_for2<PPT, false>(flags, path);
}
template <int PPT>
static void *double_kernel_for(int flags) {
    const bool nf = flags & IDIWF_NF, sc = flags & IDIWF_SCALE, so = flags & IDIWF_SECONDORDER;
    if (nf && (flags & IDIWF_ACCURATE))
        return sc ? (void *)fwd_double_kernel<PPT, true, true, false, true>
                  : (void *)fwd_double_kernel<PPT, true, false, false, true>;
    if (nf) return sc ? (void *)fwd_double_kernel<PPT, true, true, false> : (void *)fwd_double_kernel<PPT, true, false, false>;
    if (so) return sc ? (void *)fwd_double_kernel<PPT, false, true, true> : (void *)fwd_double_kernel<PPT, false, false, true>;
    return sc ? (void *)fwd_double_kernel<PPT, false, true, false> : (void *)fwd_double_kernel<PPT, false, false, false>;
}
static void *kernel_for(int precision, int ppt, int flags, bool chunked, int path = kPathRuns) {
    if (precision == IDIWF_SPLIT) {
        if (ppt == 2) return split_kernel_for<2>(flags, chunked, path);
        if (ppt == 4) return split_kernel_for<4>(flags, chunked, path);
        return split_kernel_for<8>(flags, chunked, path);
    }
    if (ppt == 1) return double_kernel_for<1>(flags);
    if (ppt == 2) return double_kernel_for<2>(flags);
    return double_kernel_for<4>(flags);
}

static idiwf_status ensure_smem(void *fn, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<void *, int>, size_t> done;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    auto key = std::make_pair(fn, dev);
    auto it = done.find(key);
    if (it != done.end() && it->second >= bytes) return IDIWF_OK;
    IDIWF_CUDA_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    done[key] = bytes;
    return IDIWF_OK;
}

// CTAs of `fn` that fit on one SM at this shape (cached per device).  The
// persistent grid never exceeds SMs x this: a CTA that only starts after the
// queue has drained would do no work and report a zero busy time.
static int resident_ctas(void *fn, int threads, size_t smem) {
    static std::mutex mu;
    static std::map<std::tuple<void *, int, int, size_t>, int> done;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    const auto key = std::make_tuple(fn, dev, threads, smem);
    auto it = done.find(key);
    if (it != done.end()) return it->second;
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        occ = 1;
    }
    occ = std::max(occ, 1);
    done[key] = occ;
    return occ;
}

// Launch the forward for images [i0, i1) of the batch (records of the whole
// batch are laid out by `rec_base`).
static idiwf_status launch_chunk(const idiwf_geom *geom, const idiwf_batch *b, int precision,
                                 int out_kind, void *out, void *ws, const LaunchShape &s,
                                 int i0, int i1, const std::vector<int64_t> &rec_base, int64_t nrec,
                                 int ksplit, cudaStream_t stream) {
    const GeomParams g = make_geom(geom);
    const int npix = geom->nx * geom->ny;
    const int tile_px = s.threads * s.ppt;
    static thread_local BatchParams bp;  // ~13 KB: keep off the stack
    std::memset(&bp, 0, sizeof(bp));
    bp.n_images = i1 - i0;
    bp.tiles_per_image = (npix + tile_px - 1) / tile_px;
    bp.te = s.te;
    if (precision != IDIWF_SPLIT) ksplit = 1;
    bp.ksplit = ksplit;
    bp.groups = precision == IDIWF_SPLIT && s.groups && geom->ny % kRun == 0;
    bp.total_units = bp.n_images * bp.tiles_per_image * ksplit;
    int max_tiles = 0;
    std::vector<int> ord(bp.n_images);
    for (int i = 0; i < bp.n_images; ++i) {
        const int64_t n = b->offsets[i0 + i + 1] - b->offsets[i0 + i];
        bp.img[i].src = b->offsets[i0 + i];
        bp.img[i].rec = rec_base[i0 + i];
        bp.img[i].n = (int32_t)n;
        bp.img[i].ntiles = (int32_t)((n + s.te - 1) / s.te);
        const int64_t nblk = (n + kChunkEmitters - 1) / kChunkEmitters;
        bp.img[i].tpc = (int32_t)((nblk + ksplit - 1) / ksplit * (kChunkEmitters / s.te));
        max_tiles = std::max(max_tiles, bp.img[i].ntiles);
        ord[i] = i;
    }
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int c) { return bp.img[a].n > bp.img[c].n; });
    for (int i = 0; i < bp.n_images; ++i) bp.order[i] = (uint16_t)ord[i];

    WsHeader *hdr = static_cast<WsHeader *>(ws);
    uint64_t *cta_ns = reinterpret_cast<uint64_t *>(static_cast<char *>(ws) + kWsTimingOffset);
    void *out_chunk = static_cast<char *>(out) +
                      (size_t)i0 * npix * (out_kind == IDIWF_OUT_C128 ? 16 : (out_kind == IDIWF_OUT_I32 ? 4 : 8));

    // prep
    if (precision == IDIWF_SPLIT)
        IDIWF_CUDA_CHECK(cudaMemsetAsync(split_recs(ws, nrec).rmax2, 0, sizeof(uint32_t) * bp.n_images, stream));
    if (max_tiles > 0) {
        dim3 pgrid((unsigned)std::min<int64_t>(((int64_t)max_tiles * s.te + 255) / 256, 1024), bp.n_images);
        if (precision == IDIWF_SPLIT) {
            const int w_mode = (geom->flags & IDIWF_NF) ? 1 : ((geom->flags & IDIWF_SECONDORDER) ? 2 : 0);
            // emitter coordinates must keep |q.r| inside the magic binade
            const double max_abs = kMaxTurns / (3.0 * 2.0 * geom->k * kInvTwoPi);
            prep_split_kernel<<<pgrid, 256, 0, stream>>>(bp, b->atoms, b->amplitudes, b->amp_dtype, w_mode,
                                                         max_abs, split_recs(ws, nrec), &hdr->error);
        } else {
            prep_double_kernel<<<pgrid, 256, 0, stream>>>(bp, b->atoms, b->amplitudes, b->amp_dtype,
                                                          double_recs(ws, nrec));
        }
        IDIWF_CUDA_CHECK(cudaGetLastError());
    }
    IDIWF_CUDA_CHECK(cudaMemsetAsync(&hdr->work_counter, 0, sizeof(uint32_t), stream));

    auto grid_for = [&](void *fn, size_t smem, int &grid) -> idiwf_status {
        idiwf_status st = ensure_smem(fn, smem);
        if (st != IDIWF_OK) return st;
        const int per_sm = std::min(s.ctas_per_sm, resident_ctas(fn, s.threads, smem));
        grid = (int)std::min<int64_t>(std::min<int64_t>(bp.total_units, (int64_t)sm_count() * per_sm), kMaxCtas);
        return IDIWF_OK;
    };
    if (precision == IDIWF_SPLIT) {
        SplitRecs rec = split_recs(ws, nrec);
        double2 *partials = ksplit > 1 ? reinterpret_cast<double2 *>(static_cast<char *>(ws) + kWsDataOffset +
                                                                     split_recs_bytes(nrec))
                                       : nullptr;
        void *args[] = {&bp, (void *)&g, &rec, &out_chunk, &out_kind, &hdr, &cta_ns, &partials};
        // the pixel-run kernel, the per-pixel kernel for the images beyond the
        // runs' bound, and in the near field the exact kernel (each returns at
        // once when it has no image)
        IDIWF_CUDA_CHECK(cudaMemsetAsync(&hdr->work_counter2, 0, 2 * sizeof(uint32_t), stream));  // + work_counter3
        for (const int path : {kPathRuns, kPathPixel, kPathExact}) {
            if (path == kPathRuns && !bp.groups) continue;
            if (path == kPathExact && !(geom->flags & IDIWF_NF)) continue;
            void *fn = kernel_for(precision, s.ppt, geom->flags, ksplit > 1, path);
            const size_t smem = fwd_smem(precision, s, path);
            int grid = 0;
            idiwf_status st = grid_for(fn, smem, grid);
            if (st != IDIWF_OK) return st;
            IDIWF_CUDA_CHECK(cudaLaunchKernel(fn, dim3(grid), dim3(s.threads), args, smem, stream));
        }
        if (ksplit > 1) {
            const int64_t total = (int64_t)bp.n_images * npix;
            const int blocks = (int)std::min<int64_t>((total + 255) / 256, 8 * (int64_t)sm_count());
            const bool nf = geom->flags & IDIWF_NF, sc = geom->flags & IDIWF_SCALE;
            if (nf)
                fwd_finish_kernel<true, false><<<blocks, 256, 0, stream>>>(g, partials, ksplit, bp.n_images,
                                                                           out_chunk, out_kind);
            else if (sc)
                fwd_finish_kernel<false, true><<<blocks, 256, 0, stream>>>(g, partials, ksplit, bp.n_images,
                                                                           out_chunk, out_kind);
            else
                fwd_finish_kernel<false, false><<<blocks, 256, 0, stream>>>(g, partials, ksplit, bp.n_images,
                                                                            out_chunk, out_kind);
            IDIWF_CUDA_CHECK(cudaGetLastError());
        }
    } else {
        DoubleRecs rec = double_recs(ws, nrec);
        void *args[] = {&bp, (void *)&g, &rec, &out_chunk, &out_kind, &hdr, &cta_ns};
        void *fn = kernel_for(precision, s.ppt, geom->flags, false);
        const size_t smem = fwd_smem(precision, s, kPathPixel);
        int grid = 0;
        idiwf_status st = grid_for(fn, smem, grid);
        if (st != IDIWF_OK) return st;
        IDIWF_CUDA_CHECK(cudaLaunchKernel(fn, dim3(grid), dim3(s.threads), args, smem, stream));
    }
    return IDIWF_OK;
}

static idiwf_status forward_impl(const idiwf_geom *geom, const idiwf_batch *b, int precision,
                                 int out_kind, void *out, void *ws, size_t ws_bytes,
                                 const LaunchShape &s, cudaStream_t stream) {
    const size_t need = forward_ws_bytes(geom, b, precision, s);
    if (!ws || ws_bytes < need)
        return set_error(IDIWF_ERR_WORKSPACE, "workspace smaller than idiwf_forward_workspace_size()");
    if (reinterpret_cast<uintptr_t>(ws) & 255) return set_error(IDIWF_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    std::vector<int64_t> rec_base(b->n_images + 1, 0);
    for (int i = 0; i < b->n_images; ++i) {
        const int64_t n = b->offsets[i + 1] - b->offsets[i];
        rec_base[i + 1] = rec_base[i] + (n + s.te - 1) / s.te * s.te;
    }
    const int64_t nrec = std::max<int64_t>(rec_base[b->n_images], 1);
    // reset the work counter and the error word: errors reported by
    // idiwf_workspace_error() are those of the most recent call
    IDIWF_CUDA_CHECK(cudaMemsetAsync(ws, 0, 2 * sizeof(uint32_t), stream));
    const int ksplit = precision == IDIWF_SPLIT ? choose_ksplit(geom, b) : 1;
    for (int i0 = 0; i0 < b->n_images; i0 += kMaxImagesPerLaunch) {
        const int i1 = std::min(b->n_images, i0 + kMaxImagesPerLaunch);
        idiwf_status st =
            launch_chunk(geom, b, precision, out_kind, out, ws, s, i0, i1, rec_base, nrec, ksplit, stream);
        if (st != IDIWF_OK) return st;
    }
    return IDIWF_OK;
}

}  // namespace idiwf

using namespace idiwf;

extern "C" size_t idiwf_forward_workspace_size(const idiwf_geom *geom, const idiwf_batch *batch,
                                               int32_t precision, const idiwf_config *cfg) {
    if (validate_geom(geom) != IDIWF_OK || validate_batch(batch) != IDIWF_OK) return 0;
    if (precision != IDIWF_SPLIT && precision != IDIWF_DOUBLE) return 0;
    // size for the largest tile any shape may use, so a tuned shape always fits
    LaunchShape s;
    if (resolve_shape(geom, batch, precision, cfg, s) != IDIWF_OK) return 0;
    LaunchShape big = s;
    big.te = 1024;
    return std::max(forward_ws_bytes(geom, batch, precision, s), forward_ws_bytes(geom, batch, precision, big));
}

extern "C" idiwf_status idiwf_forward(const idiwf_geom *geom, const idiwf_batch *batch, int32_t precision,
                                      int32_t out_kind, void *out, void *workspace, size_t workspace_bytes,
                                      const idiwf_config *cfg, cudaStream_t stream) {
    idiwf_status st = validate_geom(geom);
    if (st != IDIWF_OK) return st;
    if ((st = validate_batch(batch)) != IDIWF_OK) return st;
    if (precision != IDIWF_SPLIT && precision != IDIWF_DOUBLE)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "precision must be IDIWF_SPLIT or IDIWF_DOUBLE");
    if (out_kind < IDIWF_OUT_C128 || out_kind > IDIWF_OUT_I32)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "unknown out_kind");
    if (!out) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "out is NULL");
    LaunchShape s;
    if ((st = resolve_shape(geom, batch, precision, cfg, s)) != IDIWF_OK) return st;
    return forward_impl(geom, batch, precision, out_kind, out, workspace, workspace_bytes, s, stream);
}

extern "C" idiwf_status idiwf_forward_cta_times(const void *workspace, uint64_t *host_ns, int32_t cap,
                                                int32_t *n, cudaStream_t stream) {
    if (!workspace || !host_ns || !n || cap <= 0) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "bad arguments");
    WsHeader h;
    IDIWF_CUDA_CHECK(cudaMemcpyAsync(&h, workspace, sizeof(h), cudaMemcpyDeviceToHost, stream));
    IDIWF_CUDA_CHECK(cudaStreamSynchronize(stream));
    const int cnt = std::min<int>((int)h.n_ctas, std::min(cap, kMaxCtas));
    if (cnt > 0)
        IDIWF_CUDA_CHECK(cudaMemcpyAsync(host_ns, static_cast<const char *>(workspace) + kWsTimingOffset,
                                         sizeof(uint64_t) * cnt, cudaMemcpyDeviceToHost, stream));
    IDIWF_CUDA_CHECK(cudaStreamSynchronize(stream));
    *n = cnt;
    return IDIWF_OK;
}

extern "C" idiwf_status idiwf_tune(const idiwf_geom *geom, const idiwf_batch *batch, int32_t precision,
                                   int32_t out_kind, void *out, void *workspace, size_t workspace_bytes,
                                   cudaStream_t stream, idiwf_config *best) {
    idiwf_status st = validate_geom(geom);
    if (st != IDIWF_OK) return st;
    if ((st = validate_batch(batch)) != IDIWF_OK) return st;
    if (precision != IDIWF_SPLIT && precision != IDIWF_DOUBLE)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "precision must be IDIWF_SPLIT or IDIWF_DOUBLE");
    std::vector<LaunchShape> cands;
    if (precision == IDIWF_SPLIT) {
        // CTAs per SM: as many as fit.  The persistent queue balances any grid,
        // and a small tuning batch would favour fewer CTAs only through its
        // own last-wave tail.
        for (int th : {128, 256})
            for (int ppt : {2, 4, 8})
                for (int te : {256, 512}) {
                    LaunchShape c{th, ppt, te, 1};
                    void *fn = kernel_for(precision, ppt, geom->flags, false);
                    const size_t smem = fwd_smem(precision, c, kPathRuns);
                    if (ensure_smem(fn, smem) != IDIWF_OK) continue;
                    c.ctas_per_sm = std::min(8, resident_ctas(fn, th, smem));
                    cands.push_back(c);
                }
    } else {
        for (int th : {128, 256})
            for (int ppt : {1, 2})
                for (int te : {64, 128}) cands.push_back(LaunchShape{th, ppt, te, 2});
    }
    // Time each shape on the whole batch (the caller sizes the batch it tunes
    // on; one warm-up + best of two timed runs per shape).
    cudaEvent_t e0, e1;
    IDIWF_CUDA_CHECK(cudaEventCreate(&e0));
    IDIWF_CUDA_CHECK(cudaEventCreate(&e1));
    float best_ms = 1e30f;
    LaunchShape best_s = default_shape(precision);
    for (const LaunchShape &s : cands) {
        if (forward_ws_bytes(geom, batch, precision, s) > workspace_bytes) continue;
        {  // more CTAs per SM than fit would only repeat a smaller candidate
            void *fn = kernel_for(precision, s.ppt, geom->flags, false);
            const size_t smem = fwd_smem(precision, s, kPathRuns);
            if (ensure_smem(fn, smem) == IDIWF_OK && s.ctas_per_sm > resident_ctas(fn, s.threads, smem)) continue;
        }
        st = forward_impl(geom, batch, precision, out_kind, out, workspace, workspace_bytes, s, stream);
        if (st != IDIWF_OK) break;
        float ms_best = 1e30f;
        for (int rep = 0; rep < 2; ++rep) {
            cudaEventRecord(e0, stream);
            st = forward_impl(geom, batch, precision, out_kind, out, workspace, workspace_bytes, s, stream);
            cudaEventRecord(e1, stream);
            if (st != IDIWF_OK) break;
            cudaEventSynchronize(e1);
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            ms_best = std::min(ms_best, ms);
        }
        if (st != IDIWF_OK) break;
        if (ms_best < best_ms) {
            best_ms = ms_best;
            best_s = s;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != IDIWF_OK) return st;
    IDIWF_CUDA_CHECK(cudaGetLastError());
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[TuneKey{precision, geom->flags, geom->nx, geom->ny, n_bucket(batch)}] = best_s;
    }
    if (best) {
        best->threads = best_s.threads;
        best->pixels_per_thread = best_s.ppt;
        best->emitters_per_tile = best_s.te;
        best->ctas_per_sm = best_s.ctas_per_sm;
        best->pixel_groups = best_s.groups ? 1 : -1;
    }
    return IDIWF_OK;
}

// ---------------------------------------------------------------------------
// Split-precision forward for callers that cannot allocate device memory.
//
// Some hosts of this library cannot call cudaMalloc at all: code that runs
// inside another framework's memory pool or allocator hooks, inside a stream
// capture they do not own, or in plug-ins whose host forbids device
// allocation.  For them this entry point keeps its scratch (work counters,
// error word, per-CTA timing, emitter tile records) in one file-scope device
// array of fixed size, so the caller passes only inputs and outputs and no
// device memory is allocated.  The host side uses no heap either: the launch
// descriptor is a static buffer, used under a mutex for the few microseconds
// it takes to build it and enqueue the launches (kernel arguments are copied
// at launch).
// ---------------------------------------------------------------------------
namespace idiwf {

static __device__ __align__(256) unsigned char g_noalloc_scratch[IDIWF_NOALLOC_SCRATCH_BYTES];

constexpr int kNoAllocMaxDevices = 64;
static std::mutex g_noalloc_mu;
static void *g_noalloc_ptr[kNoAllocMaxDevices];
static BatchParams g_noalloc_bp;  // guarded by g_noalloc_mu

// Device address of the scratch array on the current device.  The name
// g_noalloc_scratch in host code is only a host-side stand-in, so the
// address is looked up once per device (with that device current) and
// cached.  The caller holds g_noalloc_mu.
static idiwf_status noalloc_scratch_locked(void **ptr) {
    int dev = 0;
    IDIWF_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        return set_error(IDIWF_ERR_UNSUPPORTED, "idiwf_forward_noalloc: device ordinal out of range");
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_noalloc_ptr[dev] = p;
    }
    *ptr = g_noalloc_ptr[dev];
    return IDIWF_OK;
}

}  // namespace idiwf

extern "C" idiwf_status idiwf_forward_noalloc(const idiwf_geom *geom, const idiwf_batch *batch, int32_t out_kind,
                                              void *out, cudaStream_t stream) {
    idiwf_status st = validate_geom(geom);
    if (st != IDIWF_OK) return st;
    if ((st = validate_batch(batch)) != IDIWF_OK) return st;
    if (out_kind < IDIWF_OUT_C128 || out_kind > IDIWF_OUT_I32)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "unknown out_kind");
    if (!out) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "out is NULL");
    if (batch->n_images > kMaxImagesPerLaunch)
        return set_error(IDIWF_ERR_UNSUPPORTED, "idiwf_forward_noalloc: at most 512 images per call");

    const LaunchShape s{256, 4, 256, 2};
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    BatchParams &bp = g_noalloc_bp;
    std::memset(&bp, 0, sizeof(bp));
    const int npix = geom->nx * geom->ny;
    const int tile_px = s.threads * s.ppt;
    bp.n_images = batch->n_images;
    bp.tiles_per_image = (npix + tile_px - 1) / tile_px;
    bp.te = s.te;
    bp.total_units = bp.n_images * bp.tiles_per_image;
    bp.groups = geom->ny % kRun == 0;
    int64_t nrec = 0;
    int max_tiles = 0;
    for (int i = 0; i < bp.n_images; ++i) {
        const int64_t n = batch->offsets[i + 1] - batch->offsets[i];
        bp.img[i].src = batch->offsets[i];
        bp.img[i].rec = nrec;
        bp.img[i].n = (int32_t)n;
        bp.img[i].ntiles = (int32_t)((n + s.te - 1) / s.te);
        nrec += (int64_t)bp.img[i].ntiles * s.te;
        max_tiles = std::max(max_tiles, bp.img[i].ntiles);
    }
    nrec = std::max<int64_t>(nrec, 1);
    if (kWsDataOffset + split_recs_bytes(nrec) > (size_t)IDIWF_NOALLOC_SCRATCH_BYTES)
        return set_error(IDIWF_ERR_UNSUPPORTED,
                         "idiwf_forward_noalloc: batch needs more than the 16 MiB static scratch "
                         "(at most 321792 emitters in total after padding every image to a multiple of 256); "
                         "use idiwf_forward with a caller workspace");
    // images by descending emitter count (stable insertion sort, no heap)
    for (int i = 0; i < bp.n_images; ++i) {
        int j = i;
        while (j > 0 && bp.img[bp.order[j - 1]].n < bp.img[i].n) {
            bp.order[j] = bp.order[j - 1];
            --j;
        }
        bp.order[j] = (uint16_t)i;
    }

    void *ws = nullptr;
    if ((st = noalloc_scratch_locked(&ws)) != IDIWF_OK) return st;
    WsHeader *hdr = static_cast<WsHeader *>(ws);
    uint64_t *cta_ns = reinterpret_cast<uint64_t *>(static_cast<char *>(ws) + kWsTimingOffset);
    SplitRecs rec = split_recs(ws, nrec);
    const GeomParams g = make_geom(geom);

    // every call starts from zero work counters and a zero error word; the
    // records are rewritten in full by the prep kernel
    IDIWF_CUDA_CHECK(cudaMemsetAsync(ws, 0, 6 * sizeof(uint32_t), stream));  // counters 1-3, error word, n_ctas
    IDIWF_CUDA_CHECK(cudaMemsetAsync(rec.rmax2, 0, sizeof(uint32_t) * bp.n_images, stream));
    if (max_tiles > 0) {
        const int w_mode = (geom->flags & IDIWF_NF) ? 1 : ((geom->flags & IDIWF_SECONDORDER) ? 2 : 0);
        const double max_abs = kMaxTurns / (3.0 * 2.0 * geom->k * kInvTwoPi);
        dim3 pgrid((unsigned)std::min<int64_t>(((int64_t)max_tiles * s.te + 255) / 256, 1024), bp.n_images);
        prep_split_kernel<<<pgrid, 256, 0, stream>>>(bp, batch->atoms, batch->amplitudes, batch->amp_dtype, w_mode,
                                                     max_abs, rec, &hdr->error);
        IDIWF_CUDA_CHECK(cudaGetLastError());
    }
    double2 *no_partials = nullptr;  // bp.ksplit == 0: the kernels write the outputs themselves
    void *args[] = {&bp, (void *)&g, &rec, &out, &out_kind, &hdr, &cta_ns, &no_partials};
    // the pixel-run, per-pixel and (near field) exact kernels, each returning
    // at once without images; the persistent grid is clamped to the CTAs that
    // fit at once, as in idiwf_forward
    for (const int path : {kPathRuns, kPathPixel, kPathExact}) {
        if (path == kPathRuns && !bp.groups) continue;
        if (path == kPathExact && !(geom->flags & IDIWF_NF)) continue;
        void *fn = split_kernel_for<4>(geom->flags, false, path);
        const size_t smem = fwd_smem(IDIWF_SPLIT, s, path);
        IDIWF_CUDA_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int occ = 0;
        IDIWF_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, s.threads, smem));
        const int per_sm = std::max(1, std::min(s.ctas_per_sm, occ));
        const int grid = (int)std::min<int64_t>(std::min<int64_t>(bp.total_units, (int64_t)sm_count() * per_sm),
                                                kMaxCtas);
        IDIWF_CUDA_CHECK(cudaLaunchKernel(fn, dim3(grid), dim3(s.threads), args, smem, stream));
    }
    return IDIWF_OK;
}

// Error word of the most recent idiwf_forward_noalloc call on the current
// device, read from the static scratch into a stack variable (no allocation;
// the read waits for `stream`).  Same bits and statuses as
// idiwf_workspace_error.
extern "C" idiwf_status idiwf_forward_noalloc_error(cudaStream_t stream) {
    void *ws = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        idiwf_status st = noalloc_scratch_locked(&ws);
        if (st != IDIWF_OK) return st;
    }
    return idiwf_workspace_error(ws, stream);
}
