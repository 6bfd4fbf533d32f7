// Adjoint (backward) emitter-wavefield direct sum for sm_100a, split precision.
//
// For I_p = |E_p|^2 and an upstream gradient g_p = dL/dI_p the adjoint is a
// second direct sum, reduced over pixels for every emitter j:
//   G_p    = 2 g_p conj(E_p)                      (per pixel, prep kernel)
//   z_pj   = G_p exp(i phi_pj)
//   dL/da_j   =  sum_p w_pj Re z_pj
//   dL/dpsi_j = -a_j sum_p w_pj Im z_pj
//   dL/dr_j   = -a_j sum_p w_pj Im z_pj grad_r phi_pj
// with grad_r phi = -q_p + kappa_p P_p r_j in the near field (q_p = k (dhat_p -
// zhat), kappa_p = k/|d_p|, P_p = I - dhat_p dhat_p^T; the next order is
// k r^2/|d|^2, ~1e-10 relative), -q_p in the far field, plus kappa_p (x, y, 0)
// for the far-field second-order term.  The near-field projector is taken
// paraxially, P ~ diag(1, 1, 0): the kappa term is itself r / (|d| theta) of
// the main term and the neglected part is theta times that, i.e. about r/|d|
// of the gradient; images with (r/|d|)^2 > kAdjRho2, or whose phase needs the
// forward's exact near-field remainder, take the exact adjoint instead:
//   grad_r phi = -q_p + (k/L) ((N - s) dhat_p + r_j),  L = |d_p - r_j|,
// with N and s as in the forward, and for "scale" grad_r (1/L) = (d_p - r_j)/L^3
// (the paraxial path uses the gradient dhat_p/|d_p|^2 of its own 1/r factor).
//
// The phase is formed as in the forward split kernel (FP64 turns in a magic
// binade -> 32-bit fixed point -> FP32 angle, MUFU sincos), with the
// pixel's constant near-field phase folded into G instead of the per-pair
// chain.  Here each
// thread owns a few emitters in registers and pixel tiles stream through
// shared memory (bulk async copies, double-buffered, bounded waits); packed
// f32x2 arithmetic processes two emitters per instruction.  Work units are
// (image, emitter block, pixel chunk); each unit writes FP32 partial sums of
// its 2048-pixel chunk, and a reduction kernel adds the chunks in a fixed
// order in FP64, so results are deterministic.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "idiwf_internal.cuh"

namespace idiwf {

constexpr int kBwdThreads = 128;
constexpr int kBwdTP = 128;                      // pixels per shared-memory tile
constexpr int kBwdChunk = 2048;                  // largest number of pixels per work unit
constexpr int kBwdNAcc = 6;                      // partial sums per emitter
constexpr int kBwdMaxPE = 8;                     // largest emitters-per-thread instantiation

// pixel record (geometry part, shared by all images):
//   P64  double4 {-q'x, -q'y, -q'z, 0}   q' = k (dhat - zhat) / 2pi      32 B
//   PF   float4 x5  {dx,dx,dy,dy} {dz,dz,-h,-h} {qx,qx,qy,qy} {qz,qz,kap,kap}
//                   {iD,iD,iD2,iD2}   (the last one read in "scale" mode) 80 B
// per image:
//   PG   float4 {G'r,G'r,G'i,G'i}   G' = 2 g conj(E) exp(2 pi i C')      16 B
// Values are duplicated in pairs because f32x2 instructions process two
// emitters of a thread against the same pixel.
constexpr int kPixRecBytes = 32 + 80 + 16;
// pixel runs (kRun pixels share one FP64 base phase), in addition:
//   PD   float4 x2  {Dx,Dx,Dy,Dy} {Dz,Dz,-h,-h}   D = 2 pi (nq_p - nq_base)   32 B per pixel
//   RB64 double4    {-q'x, -q'y, -q'z, 0} at the run's middle                 32 B per run
//   RBF  float4 x2  {dbx,dbx,dby,dby} {dbz,dbz,-hb,-hb}  d_hat and -k/(2|d|) at the run's middle  32 B per run
// Stage layouts (bytes): per-pixel path P64 | PF | PG; run path PF | PD | PG | RB64 | RBF.
constexpr uint32_t kStagePixels = kBwdTP * kPixRecBytes;
constexpr uint32_t kOffRunPF = 0;
constexpr uint32_t kOffRunPD = kBwdTP * 80;
constexpr uint32_t kOffRunPG = kOffRunPD + kBwdTP * 32;
constexpr uint32_t kOffRunB64 = kOffRunPG + kBwdTP * 16;
constexpr uint32_t kOffRunBF = kOffRunB64 + kBwdTP / kRun * 32;
constexpr uint32_t kStageRuns = kOffRunBF + kBwdTP / kRun * 32;
// exact near-field path: the per-pixel stage plus
//   PX   float4 {|d|, |d|, 0, 0}                                             16 B
// and the P64 record carries the quadratic term's coefficient kp/(2|d|) in .w
constexpr uint32_t kStageExact = kStagePixels + kBwdTP * 16;
constexpr uint32_t kStageMax = kStageRuns > kStageExact ? (kStageRuns > kStagePixels ? kStageRuns : kStagePixels)
                                                        : (kStageExact > kStagePixels ? kStageExact : kStagePixels);
static_assert(kBwdTP % kRun == 0 && kBwdChunk % kRun == 0, "tiles hold whole runs");

struct BwdLayout {
    int npix_pad;          // pixels rounded up to the chunk size
    int n_chunks, chunk_px;
    int64_t nrec;          // emitter records (images padded to the emitter block)
    size_t off_p64, off_pf, off_pg, off_pd, off_rb64, off_rbf, off_px, off_rmax, off_erec64, off_erecf, off_part, total;
};

// Pixels per work unit: 2048, 1024 or 512, whichever gives the shortest
// estimated makespan of the persistent adjoint -- the number of unit waves
// over the resident CTAs (4 per SM, the default shape) times the unit's
// pixels plus one tile of pipeline fill.  With few units per CTA the last
// wave runs part-empty: 10k emitters on 512^2 pixels make 20 emitter blocks x
// 128 chunks of 2048 = 4.3 waves on 592 CTAs (5 waves' time), but 8.6 of 1024
// (9).  Ties keep the larger unit (fewer partial sums).
static int bwd_chunk_px(const idiwf_geom *g, const idiwf_batch *b) {
    const int64_t npix = (int64_t)g->nx * g->ny;
    int64_t nb = 0;
    for (int i = 0; i < b->n_images; ++i) {
        const int64_t n = b->offsets[i + 1] - b->offsets[i];
        nb += (n + kBwdThreads * 4 - 1) / (kBwdThreads * 4);
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t slots = (int64_t)std::max(sms, 1) * 4;
    int best = kBwdChunk;
    int64_t best_cost = -1;
    for (const int c : {kBwdChunk, kBwdChunk / 2, kBwdChunk / 4}) {
        const int64_t units = std::max<int64_t>(nb, 1) * ((npix + c - 1) / c);
        const int64_t cost = (units + slots - 1) / slots * (c + kBwdTP);
        if (best_cost < 0 || cost < best_cost) {
            best_cost = cost;
            best = c;
        }
    }
    return best;
}

static BwdLayout bwd_layout(const idiwf_geom *g, const idiwf_batch *b) {
    BwdLayout L;
    const int64_t npix = (int64_t)g->nx * g->ny;
    const int eb = kBwdThreads * kBwdMaxPE;
    L.chunk_px = bwd_chunk_px(g, b);
    L.npix_pad = (int)((npix + L.chunk_px - 1) / L.chunk_px * L.chunk_px);
    L.n_chunks = L.npix_pad / L.chunk_px;
    L.nrec = 0;
    for (int i = 0; i < b->n_images; ++i) {
        const int64_t n = b->offsets[i + 1] - b->offsets[i];
        L.nrec += (n + eb - 1) / eb * eb;
    }
    L.nrec = std::max<int64_t>(L.nrec, eb);
    size_t o = kWsDataOffset;
    L.off_p64 = o; o += align256((size_t)L.npix_pad * 32);
    L.off_pf = o;  o += align256((size_t)L.npix_pad * 80);
    L.off_pg = o;  o += align256((size_t)L.npix_pad * 16 * b->n_images);
    L.off_pd = o;  o += align256((size_t)L.npix_pad * 32);
    L.off_rb64 = o; o += align256((size_t)L.npix_pad / kRun * 32);
    L.off_rbf = o; o += align256((size_t)L.npix_pad / kRun * 32);
    L.off_px = o;  o += align256((size_t)L.npix_pad * 16);
    L.off_rmax = o; o += align256((size_t)kMaxImagesPerLaunch * 4);
    L.off_erec64 = o; o += align256((size_t)L.nrec * 32);
    L.off_erecf = o;  o += align256((size_t)L.nrec * 16);
    L.off_part = o;   o += align256((size_t)L.n_chunks * L.nrec * kBwdNAcc * 4);
    L.total = o;
    return L;
}

struct BwdImage {
    int64_t src, rec;
    int32_t n, nblocks;
};
struct BwdParams {
    int32_t n_images, n_chunks, npix, npix_pad, total_units, eb;
    int32_t runs;      // pixel runs allowed (rows hold whole runs)
    int32_t chunk_px;  // pixels per work unit (a multiple of kBwdTP)
    BwdImage img[kMaxImagesPerLaunch];
    int32_t unit_img[kMaxImagesPerLaunch];   // images by descending emitter count
};

struct BwdRecs {
    const double4 *e64;
    const float4 *ef;
    const double4 *p64;
    const float4 *pf, *pg, *pd;
    const double4 *rb64;
    const float4 *rbf, *px;
    const uint32_t *rmax2;  // per image: max |r|^2 (float bits, rounded up)
};

__device__ __forceinline__ double nf_constant_turns(const GeomParams &g, double dx, double dy, double dz) {
    // k (|d| - d_z) / 2pi mod 1, without cancellation
    const double rho2 = dx * dx + dy * dy;
    const double D = sqrt(rho2 + dz * dz);
    const double c = g.kp * (dz > 0 ? rho2 / (D + dz) : D - dz);
    return c - rint(c);
}

// ---- pixel prep: geometry (image independent) ------------------------------
__global__ void bwd_pixel_geom_kernel(const GeomParams g, int npix, int npix_pad, int runs,
                                      double4 *__restrict__ p64, float4 *__restrict__ pf, float4 *__restrict__ pd,
                                      double4 *__restrict__ rb64, float4 *__restrict__ rbf, float4 *__restrict__ px) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix_pad; p += gridDim.x * blockDim.x) {
        const int pc = min(p, npix - 1);
        const int ix = pc / g.ny, iy = pc - ix * g.ny;
        double dx, dy, dz;
        pixel_cpu(g, ix, iy, dx, dy, dz);
        const double rho2 = dx * dx + dy * dy;
        const double D = sqrt(rho2 + dz * dz);
        const double invD = 1.0 / D;
        const double dzm1 = dz > 0 ? -rho2 / (D * (D + dz)) : dz * invD - 1.0;
        // .w: the exact path's quadratic-term coefficient kp / (2|d|)
        p64[p] = make_double4(-g.kp * (dx * invD), -g.kp * (dy * invD), -g.kp * dzm1, 0.5 * g.kp * invD);
        px[p] = make_float4((float)D, (float)D, 0.f, 0.f);
        const float fdx = (float)(dx * invD), fdy = (float)(dy * invD), fdz = (float)(dz * invD);
        const float fh = (float)(-g.k * 0.5 * invD);  // -h, pairs with the negated w
        const float qx = (float)(g.k * dx * invD), qy = (float)(g.k * dy * invD), qz = (float)(g.k * dzm1);
        const float kap = (float)(g.k * invD);
        const float fi = (float)invD, fi2 = (float)(invD * invD);
        float4 *r = pf + (size_t)p * 5;
        r[0] = make_float4(fdx, fdx, fdy, fdy);
        r[1] = make_float4(fdz, fdz, fh, fh);
        r[2] = make_float4(qx, qx, qy, qy);
        r[3] = make_float4(qz, qz, kap, kap);
        r[4] = make_float4(fi, fi, fi2, fi2);
        if (runs) {
            // the run's middle (rows hold whole runs), and this pixel's offset coefficients
            const int rs = min(p / kRun * kRun, npix - kRun);
            const int rix = rs / g.ny;
            const PixelDir b = pixel_dir(g, (double)rix, (double)(rs - rix * g.ny) + 0.5 * (kRun - 1));
            const PixelDir q = pixel_dir(g, (double)ix, (double)iy);
            const float Dx = (float)(kTwoPi * (q.nqx - b.nqx)), Dy = (float)(kTwoPi * (q.nqy - b.nqy)),
                        Dz = (float)(kTwoPi * (q.nqz - b.nqz));
            pd[(size_t)p * 2] = make_float4(Dx, Dx, Dy, Dy);
            pd[(size_t)p * 2 + 1] = make_float4(Dz, Dz, fh, fh);
            if (p % kRun == 0) {
                const int run = p / kRun;
                rb64[run] = make_double4(b.nqx, b.nqy, b.nqz, 0.0);
                const float ux = (float)b.ux, uy = (float)b.uy, uz = (float)b.uz;
                const float hb = (float)(-g.k * 0.5 * b.invD);
                rbf[(size_t)run * 2] = make_float4(ux, ux, uy, uy);
                rbf[(size_t)run * 2 + 1] = make_float4(uz, uz, hb, hb);
            }
        }
    }
}

// ---- pixel prep: G'_p = 2 g_p conj(E_p) exp(2 pi i C'_p) per image --------
// C'_p is the near-field constant phase k (|d| - d_z) that the per-pair
// phase leaves out; folding it into G keeps the per-pair FP64 chain at three
// DFMA.
template <bool NF>
__global__ void bwd_pixel_g_kernel(const GeomParams g, const double2 *__restrict__ field,
                                   const double *__restrict__ gI, int npix, int npix_pad, int n_images,
                                   float4 *__restrict__ pg) {
    const int64_t total = (int64_t)npix_pad * n_images;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(t / npix_pad);
        const int p = (int)(t - (int64_t)b * npix_pad);
        float gr = 0.f, gi = 0.f;
        if (p < npix) {
            const double2 e = field[(int64_t)b * npix + p];
            const double gg = 2.0 * gI[(int64_t)b * npix + p];
            double r = gg * e.x, i = -gg * e.y;
            if (NF) {
                const int ix = p / g.ny, iy = p - ix * g.ny;
                double dx, dy, dz;
                pixel_cpu(g, ix, iy, dx, dy, dz);
                double sn, cs;
                sincospi(2.0 * nf_constant_turns(g, dx, dy, dz), &sn, &cs);
                const double r2 = r * cs - i * sn;
                i = r * sn + i * cs;
                r = r2;
            }
            gr = (float)r;
            gi = (float)i;
        }
        pg[t] = make_float4(gr, gr, gi, gi);
    }
}

// ---- emitter prep: records padded per image to the emitter block ------------
__global__ void bwd_emitter_prep_kernel(const __grid_constant__ BwdParams bp, const double *__restrict__ atoms,
                                        double4 *__restrict__ e64, float4 *__restrict__ ef, int w_mode,
                                        uint32_t *__restrict__ rmax2) {
    const int b = blockIdx.y;
    const BwdImage d = bp.img[b];
    const int64_t nrec = (int64_t)d.nblocks * bp.eb;
    uint32_t r2max = 0;  // float bits; non-negative floats order like their bits
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nrec; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = d.rec + j;
        if (j < d.n) {
            const double4 a = reinterpret_cast<const double4 *>(atoms)[d.src + j];
            r2max = max(r2max, __float_as_uint(__double2float_ru((a.x * a.x + a.y * a.y) + a.z * a.z)));
            double psi = a.w * kInvTwoPi;
            psi = psi - rint(psi);
            // magic binade + 1/2 turn (angle = 2pi (u - 1.5)) + 2^-24 turn rounding bias
            psi = (kTurnMagic + 0.5 + 0x1p-24) + psi;
            const double w = w_mode == 1 ? (a.x * a.x + a.y * a.y) + a.z * a.z
                                         : (w_mode == 2 ? a.x * a.x + a.y * a.y : 0.0);
            e64[r] = make_double4(a.x, a.y, a.z, psi);
            ef[r] = make_float4((float)a.x, (float)a.y, (float)a.z, (float)(-w));  // w negated
        } else {
            e64[r] = make_double4(0, 0, 0, kTurnMagic);
            ef[r] = make_float4(0, 0, 0, 0);
        }
    }
    // |r|_max of the image for the pixel-run bound (zeroed by the caller)
    r2max = __reduce_max_sync(0xffffffffu, r2max);
    if ((threadIdx.x & 31) == 0 && r2max) atomicMax(&rmax2[b], r2max);
}

__device__ __forceinline__ float2 g2(float a, float b) { return make_float2(a, b); }

// ---- the adjoint direct sum --------------------------------------------------
// Accumulators per emitter (FP32 over a 2048-pixel chunk):
//   0  sum w Re z        -> dL/da
//   1  sum w Im z        -> dL/dpsi = -a * acc1
//   2-4 sum w Im z q     -> dL/dr main term
//   5  sum w Im z kappa  -> near-field / second-order correction -kappa (x, y, 0)
// The near-field correction uses the paraxial projector: grad phi =
// -q + kappa P r with P = I - dhat dhat^T ~ diag(1, 1, 0); the neglected part
// is of relative size theta (the pixel angle) times the correction, which is
// itself r / (|d| theta) of the main term, i.e. about r/|d| of the gradient
// (bounded per image by kAdjRho2).
// The exact path (PATH = kPathExact) keeps the same six sums with
//   2-4  sum [w Im z q + c dhat],  c = -w Im z (k/L) (N - s) [+ Re z |d| / L^3]
//   5    sum [w Im z k/L] [+ Re z / L^3]                    ("scale" terms in [])
// and the final gradient a (acc[2..4] - acc[5] r) uses all of r.
// One work unit (image, emitter block, pixel chunk).  PATH = kPathPixel: every
// emitter-pixel pair forms its phase with its own FP64 DFMA chain.  PATH =
// kPathRuns: one chain per emitter and run of kRun pixels at the run's middle,
// and the FP32 offset D_p . r per pixel (D_p = 2 pi (nq_p - nq_base); bounded
// per image by the caller), with s_p = d_hat_p . r = s_base - D_p.r / k for the
// near-field term.  PATH = kPathExact: per pair, with the forward exact path's
// phase (quadratic term in the FP64 chain, FP32 remainder).  NFB (pixel runs,
// near field without "scale"): the second-order term h (|r|^2 - s^2) is taken
// once per emitter and run, at the run's middle, instead of per pixel; across
// a run it changes by at most 1.5 k r^2 run_span / |d| (bounded per image by
// the caller).  Returns true when a bounded wait gave up.
template <bool NF, bool SCALE, bool SECOND, int PE, int PATH, bool NFB = false>
__device__ __forceinline__ bool bwd_unit(const BwdParams &bp, const BwdRecs &R, float *__restrict__ part,
                                         int64_t nrec, WsHeader *__restrict__ hdr, unsigned char *smem,
                                         uint64_t *bar, int *s_abort, uint32_t &issued, uint32_t &consumed,
                                         int img, int ib, int chunk, float ninvk, const GeomParams &g) {
    constexpr bool RUNS = PATH == kPathRuns;
    constexpr bool EXACT = PATH == kPathExact;
    static_assert(!EXACT || NF, "the exact path is a near-field path");
    static_assert(!NFB || (RUNS && NF && !SCALE), "the run-base near-field term is a pixel-run path without scale");
    constexpr int PH = PE / 2;
    constexpr uint32_t kStage = RUNS ? kStageRuns : (EXACT ? kStageExact : kStagePixels);
    const int tid = threadIdx.x;
    const float2 TWO_PI2 = g2(6.28318548f, 6.28318548f);
    const float2 NEG_3PI2 = g2(-9.42477796f, -9.42477796f);
    const float2 NEG_INVK2 = g2(ninvk, ninvk);
    const int eb = kBwdThreads * PE;
    const BwdImage d = bp.img[img];
    const int64_t rec0 = d.rec + (int64_t)ib * eb + tid * PE;

    double ex[PE], ey[PE], ez[PE], epsi[PE], err[EXACT ? PE : 1];  // err: (EXACT) |r|^2 in FP64
    float2 fx[PH], fy[PH], fz[PH], fw[PH];
#pragma unroll
    for (int e = 0; e < PE; ++e) {
        const double4 r = R.e64[rec0 + e];
        ex[e] = r.x; ey[e] = r.y; ez[e] = r.z; epsi[e] = r.w;
        if (EXACT) err[e] = __fma_rn(r.z, r.z, __fma_rn(r.y, r.y, r.x * r.x));
        const float4 f = R.ef[rec0 + e];
        if (e & 1) { fx[e / 2].y = f.x; fy[e / 2].y = f.y; fz[e / 2].y = f.z; fw[e / 2].y = f.w; }
        else       { fx[e / 2].x = f.x; fy[e / 2].x = f.y; fz[e / 2].x = f.z; fw[e / 2].x = f.w; }
    }
    const float kf = (float)g.k;
    float2 ac[kBwdNAcc][PH];
#pragma unroll
    for (int a = 0; a < kBwdNAcc; ++a)
#pragma unroll
        for (int q = 0; q < PH; ++q) ac[a][q] = g2(0.f, 0.f);

    const int p_begin = chunk * bp.chunk_px;
    const int nt = bp.chunk_px / kBwdTP;
    auto issue = [&](int t) {
        const uint32_t slot = issued & 1;
        unsigned char *st = smem + slot * kStage;
        const int p0 = p_begin + t * kBwdTP;
        mbar_arrive_expect_tx(&bar[slot], kStage);
        if (RUNS) {
            bulk_g2s(st + kOffRunPF, R.pf + (size_t)p0 * 5, kBwdTP * 80, &bar[slot]);
            bulk_g2s(st + kOffRunPD, R.pd + (size_t)p0 * 2, kBwdTP * 32, &bar[slot]);
            bulk_g2s(st + kOffRunPG, R.pg + (size_t)img * bp.npix_pad + p0, kBwdTP * 16, &bar[slot]);
            bulk_g2s(st + kOffRunB64, R.rb64 + p0 / kRun, kBwdTP / kRun * 32, &bar[slot]);
            bulk_g2s(st + kOffRunBF, R.rbf + (size_t)(p0 / kRun) * 2, kBwdTP / kRun * 32, &bar[slot]);
        } else {
            bulk_g2s(st, R.p64 + p0, kBwdTP * 32, &bar[slot]);
            bulk_g2s(st + kBwdTP * 32, R.pf + (size_t)p0 * 5, kBwdTP * 80, &bar[slot]);
            bulk_g2s(st + kBwdTP * 112, R.pg + (size_t)img * bp.npix_pad + p0, kBwdTP * 16, &bar[slot]);
            if (EXACT) bulk_g2s(st + kStagePixels, R.px + p0, kBwdTP * 16, &bar[slot]);
        }
        ++issued;
    };
    if (tid == 0) {
        issue(0);
        issue(1);
    }
    for (int it = 0; it < nt; ++it) {
        const uint32_t slot = consumed & 1;
        if (!mbar_wait_bounded(&bar[slot], (consumed >> 1) & 1)) {
            record_error(&hdr->error, kErrTimeout);
            *s_abort = 1;
        }
        const unsigned char *st = smem + slot * kStage;
        // one emitter pair q against pixel j: the sincos, z and the accumulators
        auto accumulate = [&](int q, float2 arg, float2 s, const float4 &F2, const float4 &F3, const float4 &GG,
                              const float4 *sf, int j) {
            float s0, c0, s1, c1;
            __sincosf(arg.x, &s0, &c0);
            __sincosf(arg.y, &s1, &c1);
            const float2 cc = g2(c0, c1), ss = g2(s0, s1);
            // z = G' e^{i phi'}: Im z = Gr s + Gi c, Re z = Gr c - Gi s
            float2 zi = __fmul2_rn(g2(GG.x, GG.y), ss);
            zi = __ffma2_rn(g2(GG.z, GG.w), cc, zi);
            if (SCALE) {
                const float4 F4 = sf[5 * j + 4];  // iD iD iD2 iD2
                const float2 w = NF ? __ffma2_rn(s, g2(F4.z, F4.w), g2(F4.x, F4.y)) : g2(F4.x, F4.y);
                float2 zr = __fmul2_rn(g2(GG.x, GG.y), cc);
                zr = __ffma2_rn(g2(-GG.z, -GG.w), ss, zr);
                zi = __fmul2_rn(zi, w);
                ac[0][q] = __ffma2_rn(zr, w, ac[0][q]);
                if (NF) {
                    // Re z grad w, grad w = dhat / |d|^2 (the gradient of w itself)
                    const float4 F0 = sf[5 * j + 0], F1 = sf[5 * j + 1];  // dx dx dy dy | dz dz
                    const float2 c = __fmul2_rn(zr, g2(F4.z, F4.w));
                    ac[2][q] = __ffma2_rn(c, g2(F0.x, F0.y), ac[2][q]);
                    ac[3][q] = __ffma2_rn(c, g2(F0.z, F0.w), ac[3][q]);
                    ac[4][q] = __ffma2_rn(c, g2(F1.x, F1.y), ac[4][q]);
                }
            } else {
                ac[0][q] = __ffma2_rn(g2(GG.x, GG.y), cc, ac[0][q]);
                ac[0][q] = __ffma2_rn(g2(-GG.z, -GG.w), ss, ac[0][q]);
            }
            ac[1][q] = __fadd2_rn(ac[1][q], zi);
            ac[2][q] = __ffma2_rn(zi, g2(F2.x, F2.y), ac[2][q]);
            ac[3][q] = __ffma2_rn(zi, g2(F2.z, F2.w), ac[3][q]);
            ac[4][q] = __ffma2_rn(zi, g2(F3.x, F3.y), ac[4][q]);
            if (NF || SECOND) ac[5][q] = __ffma2_rn(zi, g2(F3.z, F3.w), ac[5][q]);
        };
        if (RUNS) {
            const float4 *sf = reinterpret_cast<const float4 *>(st + kOffRunPF);
            const float4 *sd = reinterpret_cast<const float4 *>(st + kOffRunPD);
            const float4 *sg = reinterpret_cast<const float4 *>(st + kOffRunPG);
            const double4 *sb64 = reinterpret_cast<const double4 *>(st + kOffRunB64);
            const float4 *sbf = reinterpret_cast<const float4 *>(st + kOffRunBF);
#pragma unroll 1
            for (int rr = 0; rr < kBwdTP / kRun; ++rr) {
                const double4 B = sb64[rr];
                float2 XB2[PH], SB2[PH];
#pragma unroll
                for (int q = 0; q < PH; ++q) {
                    uint32_t lo[2];
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const int i = 2 * q + e;
                        double t = __fma_rn(B.x, ex[i], epsi[i]);
                        t = __fma_rn(B.y, ey[i], t);
                        t = __fma_rn(B.z, ez[i], t);
                        lo[e] = (uint32_t)__double2loint(t);
                    }
                    const float2 u = g2(__uint_as_float((lo[0] >> 9) | 0x3F800000u),
                                        __uint_as_float((lo[1] >> 9) | 0x3F800000u));
                    XB2[q] = __ffma2_rn(u, TWO_PI2, NEG_3PI2);
                    SB2[q] = g2(0.f, 0.f);
                    if (NF) {
                        const float4 B0 = sbf[2 * rr], B1 = sbf[2 * rr + 1];  // dbx dbx dby dby | dbz dbz -hb -hb
                        float2 sb = __fmul2_rn(g2(B0.x, B0.y), fx[q]);
                        sb = __ffma2_rn(g2(B0.z, B0.w), fy[q], sb);
                        SB2[q] = __ffma2_rn(g2(B1.x, B1.y), fz[q], sb);
                        if (NFB)  // (-hb)(s_b^2 - |r|^2) once for the run's pixels
                            XB2[q] = __ffma2_rn(g2(B1.z, B1.w), __ffma2_rn(SB2[q], SB2[q], fw[q]), XB2[q]);
                    }
                }
#pragma unroll 2
                for (int jj = 0; jj < kRun; ++jj) {
                    const int j = rr * kRun + jj;
                    const float4 D0 = sd[2 * j + 0];  // Dx Dx Dy Dy
                    const float4 D1 = sd[2 * j + 1];  // Dz Dz -h -h
                    const float4 F2 = sf[5 * j + 2];  // qx qx qy qy
                    const float4 F3 = sf[5 * j + 3];  // qz qz kap kap
                    const float4 GG = sg[j];          // G'r G'r G'i G'i
#pragma unroll
                    for (int q = 0; q < PH; ++q) {
                        if (NFB) {
                            // the run base holds the near-field term: the offset
                            // D_p . r goes straight onto the base angle
                            float2 arg = __ffma2_rn(g2(D0.x, D0.y), fx[q], XB2[q]);
                            arg = __ffma2_rn(g2(D0.z, D0.w), fy[q], arg);
                            arg = __ffma2_rn(g2(D1.x, D1.y), fz[q], arg);
                            accumulate(q, arg, g2(0.f, 0.f), F2, F3, GG, sf, j);
                            continue;
                        }
                        float2 dl = __fmul2_rn(g2(D0.x, D0.y), fx[q]);
                        dl = __ffma2_rn(g2(D0.z, D0.w), fy[q], dl);
                        dl = __ffma2_rn(g2(D1.x, D1.y), fz[q], dl);
                        float2 s = g2(0.f, 0.f);
                        if (NF && !NFB) {
                            s = __ffma2_rn(dl, NEG_INVK2, SB2[q]);
                            const float2 w2 = __ffma2_rn(s, s, fw[q]);  // s^2 - |r|^2
                            dl = __ffma2_rn(g2(D1.z, D1.w), w2, dl);
                        } else if (SECOND) {
                            dl = __ffma2_rn(g2(D1.z, D1.w), fw[q], dl);
                        }
                        accumulate(q, __fadd2_rn(XB2[q], dl), s, F2, F3, GG, sf, j);
                    }
                }
            }
        } else {
            const double4 *s64 = reinterpret_cast<const double4 *>(st);
            const float4 *sf = reinterpret_cast<const float4 *>(st + kBwdTP * 32);
            const float4 *sg = reinterpret_cast<const float4 *>(st + kBwdTP * 112);
            const float4 *spx = reinterpret_cast<const float4 *>(st + kStagePixels);
#pragma unroll 2
            for (int j = 0; j < kBwdTP; ++j) {
                const double4 P = s64[j];
                const float4 F0 = sf[5 * j + 0];  // dx dx dy dy
                const float4 F1 = sf[5 * j + 1];  // dz dz h h
                const float4 F2 = sf[5 * j + 2];  // qx qx qy qy
                const float4 F3 = sf[5 * j + 3];  // qz qz kap kap
                const float4 GG = sg[j];          // G'r G'r G'i G'i
                float2 D2 = g2(0.f, 0.f);
                if (EXACT) {
                    const float4 X = spx[j];  // |d| |d|
                    D2 = g2(X.x, X.y);
                }
#pragma unroll
                for (int q = 0; q < PH; ++q) {
                    uint32_t lo[2];
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const int i = 2 * q + e;
                        double t = __fma_rn(P.x, ex[i], epsi[i]);
                        t = __fma_rn(P.y, ey[i], t);
                        t = __fma_rn(P.z, ez[i], t);
                        if (EXACT) {
                            // s from the chain (t - Psi = kp (z - s)), quadratic term in FP64
                            const double sd = __fma_rn(-g.ikp, t - epsi[i], ez[i]);
                            t = __fma_rn(P.w, __fma_rn(-sd, sd, err[i]), t);
                        }
                        lo[e] = (uint32_t)__double2loint(t);
                    }
                    const float2 u = g2(__uint_as_float((lo[0] >> 9) | 0x3F800000u),
                                        __uint_as_float((lo[1] >> 9) | 0x3F800000u));
                    float2 arg = __ffma2_rn(u, TWO_PI2, NEG_3PI2);
                    float2 s = g2(0.f, 0.f);
                    if (NF) {
                        s = __fmul2_rn(g2(F0.x, F0.y), fx[q]);
                        s = __ffma2_rn(g2(F0.z, F0.w), fy[q], s);
                        s = __ffma2_rn(g2(F1.x, F1.y), fz[q], s);
                        const float2 w2 = __ffma2_rn(s, s, fw[q]);  // s^2 - |r|^2
                        if (EXACT) {
                            // L^2 = |d|(|d| - 2s) + |r|^2; N = r_perp^2 / (|d| + L - s);
                            // remainder (-h)(-N)(2s - N) as in the forward
                            const float2 l2 = __ffma2_rn(__ffma2_rn(s, g2(-2.f, -2.f), D2), D2,
                                                         g2(-fw[q].x, -fw[q].y));
                            const float2 y = g2(rsqrt_approx(l2.x), rsqrt_approx(l2.y));  // 1/L
                            const float2 den = __ffma2_rn(s, g2(-1.f, -1.f), __ffma2_rn(l2, y, D2));
                            const float2 nN = __fmul2_rn(w2, g2(rcp_approx(den.x), rcp_approx(den.y)));
                            arg = __ffma2_rn(__fmul2_rn(g2(F1.z, F1.w), nN), __ffma2_rn(s, g2(2.f, 2.f), nN), arg);
                            float s0, c0, s1, c1;
                            __sincosf(arg.x, &s0, &c0);
                            __sincosf(arg.y, &s1, &c1);
                            const float2 cc = g2(c0, c1), ss = g2(s0, s1);
                            float2 zi = __ffma2_rn(g2(GG.z, GG.w), cc, __fmul2_rn(g2(GG.x, GG.y), ss));
                            const float2 zr = __ffma2_rn(g2(-GG.z, -GG.w), ss, __fmul2_rn(g2(GG.x, GG.y), cc));
                            if (SCALE) zi = __fmul2_rn(zi, y);                              // w Im z
                            ac[0][q] = __ffma2_rn(zr, SCALE ? y : g2(1.f, 1.f), ac[0][q]);  // w Re z
                            ac[1][q] = __fadd2_rn(ac[1][q], zi);
                            const float2 kL = __fmul2_rn(g2(kf, kf), y);  // k / L
                            const float2 zk = __fmul2_rn(zi, kL);
                            // c = w Im z (k/L)(s - N) [+ Re z |d| / L^3]
                            float2 c = __fmul2_rn(zk, __fadd2_rn(s, nN));
                            float2 sk = zk;
                            if (SCALE) {
                                const float2 zy3 = __fmul2_rn(zr, __fmul2_rn(y, __fmul2_rn(y, y)));
                                c = __ffma2_rn(zy3, D2, c);
                                sk = __fadd2_rn(sk, zy3);
                            }
                            ac[2][q] = __ffma2_rn(c, g2(F0.x, F0.y), __ffma2_rn(zi, g2(F2.x, F2.y), ac[2][q]));
                            ac[3][q] = __ffma2_rn(c, g2(F0.z, F0.w), __ffma2_rn(zi, g2(F2.z, F2.w), ac[3][q]));
                            ac[4][q] = __ffma2_rn(c, g2(F1.x, F1.y), __ffma2_rn(zi, g2(F3.x, F3.y), ac[4][q]));
                            ac[5][q] = __fadd2_rn(ac[5][q], sk);
                            continue;
                        }
                        arg = __ffma2_rn(g2(F1.z, F1.w), w2, arg);
                    } else if (SECOND) {
                        arg = __ffma2_rn(g2(F1.z, F1.w), fw[q], arg);
                    }
                    accumulate(q, arg, s, F2, F3, GG, sf, j);
                }
            }
        }
        ++consumed;
        __syncthreads();
        if (*s_abort) return true;
        if (tid == 0 && it + 2 < nt) issue(it + 2);
    }
    // partials: part[chunk][rec][acc]
    float *dst = part + ((size_t)chunk * nrec + rec0) * kBwdNAcc;
#pragma unroll
    for (int q = 0; q < PH; ++q)
#pragma unroll
        for (int a = 0; a < kBwdNAcc; ++a) {
            dst[(2 * q) * kBwdNAcc + a] = ac[a][q].x;
            dst[(2 * q + 1) * kBwdNAcc + a] = ac[a][q].y;
        }
    return false;
}

// Two instances per geometry: EXACTK = false takes the units of images on the
// paraxial paths (pixel runs or per pair), EXACTK = true (near field only) the
// images that need the exact adjoint, each from its own work counter.  Every
// CTA classifies the images once into shared memory; the paraxial kernel,
// which every call runs, reports images outside the split kernels' range
// (kErrGeometry, their gradients are left at zero by the reduction).
template <bool NF, bool SCALE, bool SECOND, int PE, bool EXACTK>
__global__ void __launch_bounds__(kBwdThreads) bwd_split_kernel(const __grid_constant__ BwdParams bp,
                                                                const BwdRecs R, float *__restrict__ part,
                                                                int64_t nrec, WsHeader *__restrict__ hdr,
                                                                GeomParams g) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int s_unit, s_abort, s_img, s_ib;
    __shared__ uint8_t s_path[kMaxImagesPerLaunch], s_nfb[kMaxImagesPerLaunch];
    const int tid = threadIdx.x;
    bool mine = false;
    for (int i = tid; i < bp.n_images; i += blockDim.x) {
        const int path = split_path(g, R.rmax2[i], bp.runs != 0, true);
        s_path[i] = (uint8_t)path;
        // run base carries the near-field term: 1.5 k r^2 run_span / D <= kNfbPhaseTol (squared)
        const double r2 = (double)__uint_as_float(R.rmax2[i]);
        const double e = 1.5 * g.k * g.run_span * r2;
        s_nfb[i] = (uint8_t)(e * e * g.inv_dmin2 <= kNfbPhaseTol * kNfbPhaseTol);
        mine |= EXACTK ? path == kPathExact : (path == kPathPixel || path == kPathRuns);
        if (!EXACTK && path == kPathReject && blockIdx.x == 0) record_error(&hdr->error, kErrGeometry);
    }
    if (!__syncthreads_or(mine)) return;
    uint32_t *counter = EXACTK ? &hdr->work_counter3 : &hdr->work_counter;
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        s_abort = 0;
        mbar_fence_init();
    }
    __syncthreads();
    uint32_t issued = 0, consumed = 0;
    bool aborted = false;
    const float ninvk = (float)(-1.0 / g.k);

    for (;;) {
        __syncthreads();
        if (tid == 0) {
            // next unit of this kernel's images (the others' are skipped here)
            int u, img = 0, ib = 0;
            for (;;) {
                u = (int)atomicAdd(counter, 1u);
                if (u >= bp.total_units) break;
                ib = u / bp.n_chunks;
                for (int k = 0; k < bp.n_images; ++k) {
                    const int b = bp.unit_img[k];
                    if (ib < bp.img[b].nblocks) { img = b; break; }
                    ib -= bp.img[b].nblocks;
                }
                const int path = s_path[img];
                if (EXACTK ? path == kPathExact : (path == kPathPixel || path == kPathRuns)) break;
            }
            s_unit = u;
            s_img = img;
            s_ib = ib;
        }
        __syncthreads();
        const int unit = s_unit;
        if (unit >= bp.total_units) break;
        const int chunk = unit % bp.n_chunks;
        const int img = s_img, ib = s_ib;
        bool ab;
        if (EXACTK) {
            if constexpr (NF)
                ab = bwd_unit<NF, SCALE, SECOND, PE, kPathExact>(bp, R, part, nrec, hdr, smem, bar, &s_abort, issued,
                                                                 consumed, img, ib, chunk, ninvk, g);
            else
                ab = false;
        } else if (s_path[img] == kPathRuns) {
            if constexpr (NF && !SCALE) {
                if (s_nfb[img])
                    ab = bwd_unit<NF, SCALE, SECOND, PE, kPathRuns, true>(bp, R, part, nrec, hdr, smem, bar, &s_abort,
                                                                          issued, consumed, img, ib, chunk, ninvk, g);
                else
                    ab = bwd_unit<NF, SCALE, SECOND, PE, kPathRuns>(bp, R, part, nrec, hdr, smem, bar, &s_abort,
                                                                    issued, consumed, img, ib, chunk, ninvk, g);
            } else {
                ab = bwd_unit<NF, SCALE, SECOND, PE, kPathRuns>(bp, R, part, nrec, hdr, smem, bar, &s_abort, issued,
                                                                consumed, img, ib, chunk, ninvk, g);
            }
        } else {
            ab = bwd_unit<NF, SCALE, SECOND, PE, kPathPixel>(bp, R, part, nrec, hdr, smem, bar, &s_abort, issued,
                                                             consumed, img, ib, chunk, ninvk, g);
        }
        if (ab) {
            aborted = true;
            break;
        }
    }
    if (aborted && tid == 0)
        while (consumed < issued) {
            mbar_wait_bounded(&bar[consumed & 1], (consumed >> 1) & 1);
            ++consumed;
        }
}

// ---- chunk reduction + final gradients -------------------------------------
// Per image path as in the adjoint kernels: the exact path's correction
// acc[5] multiplies all of r, the paraxial one (x, y, 0); images outside the
// split range get zero gradients (the call reports kErrGeometry).
template <bool KAPPA>
__global__ void __launch_bounds__(256) bwd_reduce_kernel(const __grid_constant__ BwdParams bp,
                                                         const float *__restrict__ part, int64_t nrec,
                                                         const double *__restrict__ atoms,
                                                         const void *__restrict__ amps, int amp_dtype,
                                                         double *__restrict__ grad_atoms,
                                                         double *__restrict__ grad_amp, const GeomParams g,
                                                         const uint32_t *__restrict__ rmax2) {
    // 32 emitters per block (one per lane); the 8 warps take every 8th chunk,
    // so the partial sums of a chunk are read as 32 consecutive records; the
    // 8 warp sums are added in warp order (a fixed order: the result does not
    // depend on timing)
    __shared__ double red[8][32][kBwdNAcc + 1];
    const int b = blockIdx.y;
    const BwdImage d = bp.img[b];
    const int path = split_path(g, rmax2[b], bp.runs != 0, true);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int64_t j0 = (int64_t)blockIdx.x * 32; j0 < d.n; j0 += (int64_t)gridDim.x * 32) {
        const int64_t j = j0 + lane;
        double acc[kBwdNAcc];
#pragma unroll
        for (int a = 0; a < kBwdNAcc; ++a) acc[a] = 0.0;
        if (j < d.n && path != kPathReject) {
            const int64_t r = d.rec + j;
            for (int c = w; c < bp.n_chunks; c += 8) {
                const float *src = part + ((size_t)c * nrec + r) * kBwdNAcc;
#pragma unroll
                for (int a = 0; a < kBwdNAcc; ++a) acc[a] += (double)src[a];
            }
        }
#pragma unroll
        for (int a = 0; a < kBwdNAcc; ++a) red[w][lane][a] = acc[a];
        __syncthreads();
        if (w == 0 && j < d.n) {
            const int64_t s = d.src + j;
            if (path == kPathReject) {
                reinterpret_cast<double4 *>(grad_atoms)[s] = make_double4(0.0, 0.0, 0.0, 0.0);
                if (grad_amp) grad_amp[s] = 0.0;
            } else {
#pragma unroll
                for (int a = 0; a < kBwdNAcc; ++a) {
                    double t = red[0][lane][a];
                    for (int ww = 1; ww < 8; ++ww) t += red[ww][lane][a];
                    acc[a] = t;
                }
                const double4 at = reinterpret_cast<const double4 *>(atoms)[s];
                double aj = 1.0;
                if (amps) aj = amp_dtype == IDIWF_F32 ? (double)static_cast<const float *>(amps)[s]
                                                     : static_cast<const double *>(amps)[s];
                // dL/dr = -a sum w Im z grad(phi) [+ a sum Re z grad w] = a (Q - K (x, y, 0 or z))
                double gx = acc[2], gy = acc[3], gz = acc[4];
                if (KAPPA) {
                    gx -= acc[5] * at.x;
                    gy -= acc[5] * at.y;
                    if (path == kPathExact) gz -= acc[5] * at.z;
                }
                reinterpret_cast<double4 *>(grad_atoms)[s] = make_double4(aj * gx, aj * gy, aj * gz, -aj * acc[1]);
                if (grad_amp) grad_amp[s] = acc[0];
            }
        }
        __syncthreads();
    }
}

template <int PE, bool EX>
static void *bwd_kernel_for(bool nf, bool sc, bool so) {
    if (nf) return sc ? (void *)bwd_split_kernel<true, true, false, PE, EX> : (void *)bwd_split_kernel<true, false, false, PE, EX>;
    if (EX) return nullptr;  // the exact adjoint is a near-field path
    if (so) return sc ? (void *)bwd_split_kernel<false, true, true, PE, false> : (void *)bwd_split_kernel<false, false, true, PE, false>;
    return sc ? (void *)bwd_split_kernel<false, true, false, PE, false> : (void *)bwd_split_kernel<false, false, false, PE, false>;
}

}  // namespace idiwf

using namespace idiwf;

static idiwf_status bwd_validate(const idiwf_geom *g, const idiwf_batch *b) {
    if (!g || !b || !b->offsets || b->n_images <= 0)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "geom/batch missing or empty");
    if (g->nx <= 0 || g->ny <= 0 || (int64_t)g->nx * g->ny >= (int64_t)1 << 30)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "bad detector size");
    if (b->n_images > kMaxImagesPerLaunch)
        return set_error(IDIWF_ERR_UNSUPPORTED, "backward handles at most 512 images per call");
    if (b->offsets[0] != 0) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "offsets[0] must be 0");
    for (int i = 0; i < b->n_images; ++i)
        if (b->offsets[i + 1] < b->offsets[i]) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "offsets must be non-decreasing");
    if (b->atoms && (reinterpret_cast<uintptr_t>(b->atoms) & 31))
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "atoms must be 32-byte aligned");
    if (g->flags & ~(IDIWF_NF | IDIWF_SCALE | IDIWF_SECONDORDER | IDIWF_ACCURATE))
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "unknown geometry flag");
    return IDIWF_OK;
}

extern "C" size_t idiwf_backward_workspace_size(const idiwf_geom *geom, const idiwf_batch *batch,
                                                const idiwf_config *cfg) {
    (void)cfg;
    if (bwd_validate(geom, batch) != IDIWF_OK) return 0;
    return bwd_layout(geom, batch).total;
}

extern "C" idiwf_status idiwf_backward(const idiwf_geom *geom, const idiwf_batch *batch, const void *field,
                                       const double *grad_intensity, double *grad_atoms, double *grad_amp,
                                       void *workspace, size_t workspace_bytes, const idiwf_config *cfg,
                                       cudaStream_t stream) {
    (void)cfg;
    idiwf_status st = bwd_validate(geom, batch);
    if (st != IDIWF_OK) return st;
    if (!field || !grad_intensity || !grad_atoms)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "field, grad_intensity and grad_atoms are required");
    const BwdLayout L = bwd_layout(geom, batch);
    if (!workspace || workspace_bytes < L.total)
        return set_error(IDIWF_ERR_WORKSPACE, "workspace smaller than idiwf_backward_workspace_size()");
    if (reinterpret_cast<uintptr_t>(workspace) & 255)
        return set_error(IDIWF_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    const int64_t ntot = batch->offsets[batch->n_images];
    if (ntot == 0) return IDIWF_OK;

    char *ws = static_cast<char *>(workspace);
    WsHeader *hdr = reinterpret_cast<WsHeader *>(ws);
    double4 *p64 = reinterpret_cast<double4 *>(ws + L.off_p64);
    float4 *pf = reinterpret_cast<float4 *>(ws + L.off_pf);
    float4 *pg = reinterpret_cast<float4 *>(ws + L.off_pg);
    double4 *e64 = reinterpret_cast<double4 *>(ws + L.off_erec64);
    float4 *ef = reinterpret_cast<float4 *>(ws + L.off_erecf);
    float *part = reinterpret_cast<float *>(ws + L.off_part);
    float4 *pd = reinterpret_cast<float4 *>(ws + L.off_pd);
    double4 *rb64 = reinterpret_cast<double4 *>(ws + L.off_rb64);
    float4 *rbf = reinterpret_cast<float4 *>(ws + L.off_rbf);
    uint32_t *rmax2 = reinterpret_cast<uint32_t *>(ws + L.off_rmax);
    float4 *px = reinterpret_cast<float4 *>(ws + L.off_px);

    const GeomParams g = make_geom(geom);
    const int npix = geom->nx * geom->ny;
    const bool nf = geom->flags & IDIWF_NF, sc = geom->flags & IDIWF_SCALE, so = geom->flags & IDIWF_SECONDORDER;

    // emitters per thread: 4 (default) or 8, from cfg->pixels_per_thread
    const int pe = (cfg && cfg->pixels_per_thread) ? cfg->pixels_per_thread : 4;
    if (pe != 4 && pe != 8) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "backward emitters per thread must be 4 or 8");
    const int eb = kBwdThreads * pe;
    static thread_local BwdParams bp;
    std::memset(&bp, 0, sizeof(bp));
    bp.n_images = batch->n_images;
    bp.n_chunks = L.n_chunks;
    bp.chunk_px = L.chunk_px;
    bp.npix = npix;
    bp.npix_pad = L.npix_pad;
    bp.eb = eb;
    // pixel runs unless switched off (pixel_groups = -1) or rows do not hold whole runs
    bp.runs = !(cfg && cfg->pixel_groups < 0) && geom->ny % kRun == 0;
    int64_t rec = 0;
    int total_blocks = 0, max_blocks = 0;
    std::vector<int> ord(batch->n_images);
    for (int i = 0; i < batch->n_images; ++i) {
        const int64_t n = batch->offsets[i + 1] - batch->offsets[i];
        bp.img[i].src = batch->offsets[i];
        bp.img[i].rec = rec;
        bp.img[i].n = (int32_t)n;
        bp.img[i].nblocks = (int32_t)((n + eb - 1) / eb);
        rec += (int64_t)bp.img[i].nblocks * eb;
        total_blocks += bp.img[i].nblocks;
        max_blocks = std::max(max_blocks, bp.img[i].nblocks);
        ord[i] = i;
    }
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int c) { return bp.img[a].n > bp.img[c].n; });
    for (int i = 0; i < batch->n_images; ++i) bp.unit_img[i] = ord[i];
    bp.total_units = total_blocks * L.n_chunks;

    const int pthreads = 256;
    bwd_pixel_geom_kernel<<<(L.npix_pad + pthreads - 1) / pthreads, pthreads, 0, stream>>>(
        g, npix, L.npix_pad, bp.runs, p64, pf, pd, rb64, rbf, px);
    IDIWF_CUDA_CHECK(cudaGetLastError());
    {
        const int64_t tot = (int64_t)L.npix_pad * batch->n_images;
        const int blocks = (int)std::min<int64_t>((tot + pthreads - 1) / pthreads, 65535);
        if (nf)
            bwd_pixel_g_kernel<true><<<blocks, pthreads, 0, stream>>>(g, static_cast<const double2 *>(field),
                                                                      grad_intensity, npix, L.npix_pad,
                                                                      batch->n_images, pg);
        else
            bwd_pixel_g_kernel<false><<<blocks, pthreads, 0, stream>>>(g, static_cast<const double2 *>(field),
                                                                       grad_intensity, npix, L.npix_pad,
                                                                       batch->n_images, pg);
        IDIWF_CUDA_CHECK(cudaGetLastError());
    }
    {
        const int w_mode = nf ? 1 : (so ? 2 : 0);
        dim3 grid((unsigned)std::max(1, (max_blocks * eb + 255) / 256), batch->n_images);
        IDIWF_CUDA_CHECK(cudaMemsetAsync(rmax2, 0, sizeof(uint32_t) * batch->n_images, stream));
        bwd_emitter_prep_kernel<<<grid, 256, 0, stream>>>(bp, batch->atoms, e64, ef, w_mode, rmax2);
        IDIWF_CUDA_CHECK(cudaGetLastError());
    }
    // work counters (paraxial and exact kernels) and the error word
    IDIWF_CUDA_CHECK(cudaMemsetAsync(hdr, 0, 5 * sizeof(uint32_t), stream));
    int64_t nrec = L.nrec;
    BwdRecs R{e64, ef, p64, pf, pg, pd, rb64, rbf, px, rmax2};
    void *args[] = {&bp, &R, &part, &nrec, &hdr, (void *)&g};
    const size_t smem = 2 * (size_t)kStageMax;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // the paraxial kernel (every call), then in the near field the exact kernel;
    // each returns at once when it has no image
    for (const bool exact : {false, true}) {
        if (exact && !nf) continue;
        void *fn = exact ? (pe == 8 ? bwd_kernel_for<8, true>(nf, sc, so) : bwd_kernel_for<4, true>(nf, sc, so))
                         : (pe == 8 ? bwd_kernel_for<8, false>(nf, sc, so) : bwd_kernel_for<4, false>(nf, sc, so));
        IDIWF_CUDA_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int occ = 1;
        IDIWF_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kBwdThreads, smem));
        const int grid = (int)std::min<int64_t>(bp.total_units, (int64_t)sms * std::max(occ, 1));
        IDIWF_CUDA_CHECK(cudaLaunchKernel(fn, dim3(grid), dim3(kBwdThreads), args, smem, stream));
    }
    {
        int64_t max_n = 1;
        for (int i = 0; i < batch->n_images; ++i) max_n = std::max<int64_t>(max_n, bp.img[i].n);
        dim3 rgrid((unsigned)std::min<int64_t>((max_n + 31) / 32, 65535), batch->n_images);
        if (nf || so)
            bwd_reduce_kernel<true><<<rgrid, 256, 0, stream>>>(bp, part, nrec, batch->atoms, batch->amplitudes,
                                                                batch->amp_dtype, grad_atoms, grad_amp, g, rmax2);
        else
            bwd_reduce_kernel<false><<<rgrid, 256, 0, stream>>>(bp, part, nrec, batch->atoms, batch->amplitudes,
                                                                 batch->amp_dtype, grad_atoms, grad_amp, g, rmax2);
        IDIWF_CUDA_CHECK(cudaGetLastError());
    }
    return IDIWF_OK;
}
