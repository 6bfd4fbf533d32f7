// Internal declarations shared by the idiwf CUDA sources (sm_100a only).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "idiwf.h"

namespace idiwf {

// ---------------------------------------------------------------------------
// host-side error state
// ---------------------------------------------------------------------------
idiwf_status set_error(idiwf_status st, const std::string &msg);
idiwf_status cuda_error(cudaError_t e, const char *where);

#define IDIWF_CUDA_CHECK(expr)                                         \
    do {                                                               \
        cudaError_t _e = (expr);                                       \
        if (_e != cudaSuccess) return ::idiwf::cuda_error(_e, #expr);  \
    } while (0)

// ---------------------------------------------------------------------------
// constants
// ---------------------------------------------------------------------------
constexpr double kTwoPi = 6.283185307179586476925286766559;
constexpr double kInvTwoPi = 0.15915494309189533576888376337251;
// Adding 1.5*2^20 to a phase measured in turns puts it in the binade
// [2^20, 2^21) whose ulp is 2^-32: the low 32 bits of the double are then
// the fractional turn as an unsigned fixed-point number (phase mod 1).
constexpr double kTurnMagic = 1572864.0;
// Largest |phase| in turns the magic binade holds with margin.
constexpr double kMaxTurns = 262144.0;

// Workspace header (first 256 bytes of every workspace).
struct WsHeader {
    uint32_t work_counter;  // persistent-kernel work queue
    uint32_t error;         // device error word (IDIWF_ERR_* bit set)
    uint32_t n_ctas;        // CTAs of the last forward launch
    uint32_t work_counter2; // second work queue (split forward: per-pixel kernel; time path: full sorts)
    uint32_t work_counter3; // third work queue (split forward: exact near-field kernel; time path:
                            // warm-started sorts given up)
    uint32_t pad32;
    uint64_t pad[29];
};
static_assert(sizeof(WsHeader) == 256, "workspace header is 256 bytes");
constexpr int kMaxCtas = 4096;                       // per-CTA timing slots
constexpr size_t kWsTimingOffset = 256;
constexpr size_t kWsDataOffset = 256 + 8 * kMaxCtas; // 256-aligned
constexpr uint32_t kErrTimeout = 1u;
constexpr uint32_t kErrRange = 2u;
constexpr uint32_t kErrValue = 4u;  // invalid input value (negative, NaN, zero-sum, count mismatch)
// near-field image outside the split kernels' range (emitters too far out
// for the exact remainder to stay below kExactMaxPhase, or |r| > |d| / 4)
constexpr uint32_t kErrGeometry = 8u;

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Maximum images per launch (descriptors travel as kernel parameters).
constexpr int kMaxImagesPerLaunch = 512;

// Pixel runs of the split kernels: aligned blocks of kRun pixels along a
// detector row share one FP64 base phase, taken at the middle of the run.
constexpr int kRun = 4;
// Largest phase offset (radians) that a run adds in FP32 to its base phase,
// bounded per image by k * run_span * |r|_max.  Up to 1 rad the FP32 offset is
// good to about 1e-7 rad and the sine/cosine arguments stay within 1 rad of
// the base angle's range.
constexpr double kGroupMaxPhase = 1.0;

// Near field in the split kernels.  With s = d_hat . r, r_perp^2 = |r|^2 - s^2
// and L = |d - r|, the path difference is exactly
//   |d - r| - |d| = -s + N,   N = r_perp^2 / (|d| + L - s)
// (no cancellation: the denominator is about 2|d|).  The split kernels use
// N ~ r_perp^2 / (2|d|) where the dropped remainder
//   R = N - r_perp^2/(2|d|) = r_perp^2 (2s - N) / (2|d| (|d| + L - s))
// stays below kNfPhaseTol (radians, times k) for every emitter of the image.
// |R| <= r^3/(3 sqrt3 D (D-r)) + r^4/(8 D (D-r)^2) for |r| <= r, |d| >= D; with
// r <= D/4 this is at most kNfBoundC r^3 / D^2, which the classifier below
// evaluates squared (no square root in the kernels' prologues).
// Images above the tolerance take the exact near-field kernel: the quadratic
// term k r_perp^2 / (2|d|) joins the FP64 turn chain and the remainder R is
// added in FP32 from the exact expression, which needs k|R| <= kExactMaxPhase
// so that FP32 keeps it to ~1e-7 rad; beyond that (or |r| > D/4) the image is
// rejected (kErrGeometry).
constexpr double kNfPhaseTol = 1e-7;
constexpr double kExactMaxPhase = 2.0;
constexpr double kNfBoundC = 0.3122;
// "scale": the per-pixel path's 1/|d - r| ~ (1 + s/|d|)/|d| is off by at most
// (r/D)^2 relative; above kNfScaleRho2 the image takes the exact kernel
// (which forms 1/|d - r| with a reciprocal square root).
constexpr double kNfScaleRho2 = 1e-7;
// The adjoint's paraxial near-field gradient -q + k (x, y, 0)/|d| is off by
// about r/D relative; above kAdjRho the image takes the exact adjoint.
constexpr double kAdjRho2 = 1e-12;
// The adjoint's pixel runs may take the near-field term h (|r|^2 - s^2) once
// per run, at its middle, when its change across the run, at most
// 1.5 k r^2 run_span / D, stays below this (radians): about the split
// kernels' own per-pair phase rounding (1.5e-7 rad rms).
constexpr double kNfbPhaseTol = 4e-7;

// Paths of the split kernels, chosen per image from |r|_max.
constexpr int kPathPixel = 0;   // FP64 phase per pair, second-order near field
constexpr int kPathRuns = 1;    // FP64 phase per run of kRun pixels + FP32 offsets
constexpr int kPathExact = 2;   // near field with the exact remainder (per pair)
constexpr int kPathReject = 3;  // outside the split kernels' range

struct GeomParams {
    int32_t nx, ny, flags, has_rot;
    double pixelsize, detz, k, kp, ikp;  // kp = k / 2pi, ikp = 1 / kp
    double offx, offy;
    double rot[9];
    // largest |d_hat_i - d_hat_base| between a pixel of a run of 4 along a row
    // and the run's middle: half the run's length over the detector plane's
    // distance from the origin (the angle a segment subtends bounds the chord)
    double run_span;
    // distance of the detector plane from the origin (a lower bound on every
    // pixel's |d|) and the classifier's constants derived from it
    double dmin, inv_dmin2, nf_c3;  // nf_c3 = (kNfBoundC k / dmin^2)^2
};

struct ImageDesc {
    int64_t src;    // first emitter row of the image in the caller's atoms
    int64_t rec;    // first record of the image in the padded record arrays
    int32_t n;      // emitters
    int32_t ntiles; // record tiles (n rounded up to the tile size)
    int32_t tpc;    // record tiles per emitter chunk (split over emitters)
    int32_t pad;
};

struct BatchParams {
    int32_t n_images;
    int32_t tiles_per_image;  // pixel tiles per image
    int32_t te;               // emitters per tile
    int32_t total_units;      // n_images * tiles_per_image * ksplit
    int32_t ksplit;           // emitter chunks per (image, pixel tile); 0 or 1 = none
    int32_t groups;           // split forward: phase per pixel run + FP32 offsets where bounded
    ImageDesc img[kMaxImagesPerLaunch];
    uint16_t order[kMaxImagesPerLaunch];  // images by descending emitter count
};

// Emitters per chunk are a multiple of this, so chunk boundaries -- and with
// them the summation order -- do not depend on the kernel shape.
constexpr int kChunkEmitters = 1024;

GeomParams make_geom(const idiwf_geom *g);

// ---------------------------------------------------------------------------
// device helpers: mbarrier + bulk async copy into the CTA's own shared memory
// ---------------------------------------------------------------------------
#if defined(__CUDACC__)

// try_wait suspends for a hardware time window per call; this cap bounds a
// wait to a few seconds, after which the caller records kErrTimeout.
constexpr uint32_t kWaitLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: true when the phase completed, false when the cap ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
    for (uint32_t it = 0; it < kWaitLimit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Global -> shared bulk copy (size and both addresses 16-byte aligned),
// completion signalled on `bar` as transaction bytes.
__device__ __forceinline__ void bulk_g2s(void *sdst, const void *gsrc, uint32_t bytes,
                                         uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(sdst)),
        "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Detector pixel position, idi/simulation/cpu.py:76-80 rounding sequence
// (float nx/2, separate multiply and add, numba's contracted mat-vec).
// (fractional indices give points between pixel centres, e.g. the centre of a
// run of pixels)
__device__ __forceinline__ void pixel_cpu_at(const GeomParams &g, double fix, double fiy, double &x,
                                             double &y, double &z) {
    const double px = __dadd_rn(__dmul_rn(__dsub_rn(fix, g.nx * 0.5), g.pixelsize), g.offx);
    const double py = __dadd_rn(__dmul_rn(__dsub_rn(fiy, g.ny * 0.5), g.pixelsize), g.offy);
    const double pz = g.detz;
    if (g.has_rot) {
        const double *M = g.rot;
        x = __fma_rn(M[2], pz, __fma_rn(M[0], px, __dmul_rn(M[1], py)));
        y = __fma_rn(M[5], pz, __fma_rn(M[3], px, __dmul_rn(M[4], py)));
        z = __fma_rn(M[8], pz, __fma_rn(M[6], px, __dmul_rn(M[7], py)));
    } else {
        x = px;
        y = py;
        z = pz;
    }
}
__device__ __forceinline__ void pixel_cpu(const GeomParams &g, int ix, int iy, double &x,
                                          double &y, double &z) {
    pixel_cpu_at(g, (double)ix, (double)iy, x, y, z);
}

// Direction of a detector point for the split kernels: the FP64 turn
// coefficients nq = -k (d_hat - z_hat) / 2pi (z part without cancellation),
// d_hat and 1/|d|.
struct PixelDir {
    double nqx, nqy, nqz, ux, uy, uz, invD;
};
__device__ __forceinline__ PixelDir pixel_dir(const GeomParams &g, double fix, double fiy) {
    double dx, dy, dz;
    pixel_cpu_at(g, fix, fiy, dx, dy, dz);
    const double rho2 = dx * dx + dy * dy;
    const double D = sqrt(rho2 + dz * dz);
    const double invD = 1.0 / D;
    const double dzm1 = dz > 0 ? -rho2 / (D * (D + dz)) : dz * invD - 1.0;
    PixelDir p;
    p.ux = dx * invD;
    p.uy = dy * invD;
    p.uz = dz * invD;
    p.nqx = -g.kp * p.ux;
    p.nqy = -g.kp * p.uy;
    p.nqz = -g.kp * dzm1;
    p.invD = invD;
    return p;
}

// Detector pixel position, idi/simulation/time.py:77-81 (meshgrid, dets @ M.T
// as OpenBLAS evaluates it: fma(M[i,2], z, fma(M[i,1], y, M[i,0]*x))).
__device__ __forceinline__ void pixel_time(const GeomParams &g, int ix, int iy, double &x,
                                           double &y, double &z) {
    const double px = __dmul_rn(g.pixelsize, __dsub_rn((double)ix, g.nx * 0.5));
    const double py = __dmul_rn(g.pixelsize, __dsub_rn((double)iy, g.ny * 0.5));
    const double pz = g.detz;
    if (g.has_rot) {
        const double *M = g.rot;
        x = __fma_rn(M[2], pz, __fma_rn(M[1], py, __dmul_rn(M[0], px)));
        y = __fma_rn(M[5], pz, __fma_rn(M[4], py, __dmul_rn(M[3], px)));
        z = __fma_rn(M[8], pz, __fma_rn(M[7], py, __dmul_rn(M[6], px)));
    } else {
        x = px;
        y = py;
        z = pz;
    }
}

__device__ __forceinline__ void record_error(uint32_t *err, uint32_t bit) { atomicOr(err, bit); }

// Path of one image in the split kernels, from the image's max |r|^2 (float
// bits, rounded up).  `runs`: pixel runs allowed in this launch; `adjoint`:
// the backward's paraxial-gradient bound applies as well.  The choice depends
// on the image and the geometry only, so results do not depend on the kernel
// shape.  Squared comparisons throughout; a NaN |r|^2 fails the run test and
// skips the near-field tests (NaN coordinates are reported by the range check).
__device__ __forceinline__ int split_path(const GeomParams &g, uint32_t r2bits, bool runs, bool adjoint) {
    const double r2 = (double)__uint_as_float(r2bits);
    if ((g.flags & IDIWF_NF) && r2 > 0.0) {
        const double rho2 = r2 * g.inv_dmin2;
        const double t2 = g.nf_c3 * r2 * r2 * r2;  // (bound on k |R|)^2
        if (!(rho2 <= 1.0 / 16.0 && t2 <= kExactMaxPhase * kExactMaxPhase)) return kPathReject;
        const bool paraxial = t2 <= kNfPhaseTol * kNfPhaseTol &&
                              (!(g.flags & IDIWF_SCALE) || rho2 <= kNfScaleRho2) && (!adjoint || rho2 <= kAdjRho2);
        if (!paraxial) return kPathExact;
    }
    const double ks = g.k * g.run_span;
    return (runs && ks * ks * r2 <= kGroupMaxPhase * kGroupMaxPhase) ? kPathRuns : kPathPixel;
}

// Reciprocal square root and reciprocal on the MUFU pipe (relative error a
// few 2^-23; flush-to-zero, for operands of the size of detector distances).
__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

#endif  // __CUDACC__

}  // namespace idiwf
