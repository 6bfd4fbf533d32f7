/*
 * idiwf — B200 (sm_100a) emitter-wavefield direct sum, C ABI.
 *
 * The library computes, for every detector pixel p and image b,
 *     E_bp = sum_j a_j w_pj exp(i phi_pj),   I_bp = |E_bp|^2
 * over the emitters j of image b, in the geometry and phase conventions of
 * fzimmermann89/idi (idi/simulation/cpu.py, idi/simulation/sim.cu), plus the
 * time-dependent variant of idi/simulation/time.py and simtime.cu.
 *
 * Conventions shared by every entry point
 *  - Lengths in the caller's unit (the reference uses micrometres), k in 1/length.
 *  - Emitters use the reference's (N,4) float64 layout [x, y, z, phase]
 *    (idi/simulation/cuda.py:85, cpu.py:69), row-major, on the DEVICE.
 *  - Detector arrays are (nx, ny) row-major, pixel (ix, iy) at
 *    ((ix - nx/2) * pixelsize + offset[0], (iy - ny/2) * pixelsize + offset[1], detz),
 *    optionally rotated by rot (idi/simulation/cpu.py:76-80).
 *  - Every device buffer is allocated by the caller.  Scratch space is a
 *    caller-provided workspace whose size the *_workspace_size functions report;
 *    no entry point allocates device or pinned memory.
 *  - Work is enqueued on `stream` and is asynchronous: the compute entry points
 *    do not synchronise, so they can be captured in a CUDA graph.  The entry
 *    points that read results back (idiwf_tune, idiwf_forward_cta_times,
 *    idiwf_workspace_error, idiwf_microbench) synchronise their stream.
 *  - Errors are returned as idiwf_status, never by aborting.  Asynchronous
 *    device-side failures (a bounded wait that ran out) are recorded in the
 *    workspace and reported by idiwf_workspace_error().
 *  - The library holds no global mutable state except the autotune cache
 *    (mutex-protected) and a thread-local last-error string.
 */
#ifndef IDIWF_H
#define IDIWF_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t idiwf_status;
#define IDIWF_OK 0
#define IDIWF_ERR_INVALID_ARGUMENT 1
#define IDIWF_ERR_CUDA 2
#define IDIWF_ERR_WORKSPACE 3   /* workspace missing, too small or misaligned */
#define IDIWF_ERR_TIMEOUT 4     /* a bounded device-side wait gave up */
#define IDIWF_ERR_UNSUPPORTED 5 /* size or mode outside what the kernels implement */

/* geometry flags: the reference's `settings` substrings (cuda.py:51-65) */
#define IDIWF_NF 1          /* "nf": exact spherical path |d - r| (else far field) */
#define IDIWF_SCALE 2       /* "scale": 1/r amplitude factor */
#define IDIWF_SECONDORDER 4 /* "secondorder": Fresnel term of sim.cu:88 (far field) */
#define IDIWF_ACCURATE 8    /* IDIWF_DOUBLE near field: cancellation-free |d-r|-|d| instead of
                               the reference's rounding sequence (ignored elsewhere) */

/* precision */
#define IDIWF_DOUBLE 0 /* all-FP64, reproduces the reference CPU rounding sequence */
#define IDIWF_SPLIT 1  /* FP64 path difference + phase reduction, FP32 sincos/accumulation */

/* output kinds */
#define IDIWF_OUT_C128 0 /* complex128 field, interleaved (re, im) doubles */
#define IDIWF_OUT_C64 1  /* complex64 field */
#define IDIWF_OUT_I64 2  /* float64 intensity |E|^2 */
#define IDIWF_OUT_I32 3  /* float32 intensity */

/* element types of amplitude, probability and count arrays */
#define IDIWF_F64 0
#define IDIWF_F32 1
#define IDIWF_I32 2
#define IDIWF_U32 3
#define IDIWF_I64 4

typedef struct idiwf_geom {
    int32_t nx, ny;   /* detector pixels: Ndet[0] (rows), Ndet[1] (columns) */
    int32_t flags;    /* IDIWF_NF | IDIWF_SCALE | IDIWF_SECONDORDER */
    int32_t has_rot;  /* nonzero: apply rot to every pixel position */
    double pixelsize; /* pixel pitch */
    double detz;      /* detector distance */
    double k;         /* angular wavenumber 2 pi / lambda */
    double offset[2]; /* detoffset (x, y) */
    double rot[9];    /* row-major rotation from detangles (idi/util rotation(theta, phi, 0)) */
} idiwf_geom;

/* Kernel shape; zero fields select the tuned (or default) value. */
typedef struct idiwf_config {
    int32_t threads;            /* threads per CTA (split: 128 or 256) */
    int32_t pixels_per_thread;  /* split forward: 4 or 8; double forward: 2 */
    int32_t emitters_per_tile;  /* emitters staged per shared-memory tile: 64..512 */
    int32_t ctas_per_sm;        /* persistent grid = SMs * ctas_per_sm */
    int32_t pixel_groups;       /* split forward: 0 or 1 = one FP64 phase per run of pixels plus
                                   FP32 offsets wherever the offsets stay below 1 rad (checked per
                                   work unit on the device), -1 = an FP64 phase for every pixel */
} idiwf_config;

/* Batch of images with uneven emitter counts.  Image b owns emitter rows
 * [offsets[b], offsets[b+1]) of `atoms` (and of `amplitudes`). */
typedef struct idiwf_batch {
    int32_t n_images;
    int32_t amp_dtype;        /* IDIWF_F64 or IDIWF_F32; ignored when amplitudes == NULL */
    const int64_t *offsets;   /* HOST array, n_images + 1 entries, offsets[0] == 0 */
    const double *atoms;      /* DEVICE (offsets[n_images], 4) float64 [x, y, z, phase] */
    const void *amplitudes;   /* DEVICE (offsets[n_images]) or NULL for unit amplitudes */
} idiwf_batch;

/* ------------------------------------------------------------------------ */
/* forward direct sum                                                        */
/* ------------------------------------------------------------------------ */

/* Bytes of workspace idiwf_forward needs for this batch (256-byte aligned base). */
size_t idiwf_forward_workspace_size(const idiwf_geom *geom, const idiwf_batch *batch,
                                    int32_t precision, const idiwf_config *cfg);

/*
 * Forward direct sum of every image of `batch` into `out`
 * ((n_images, nx, ny) of `out_kind`), in one persistent launch whose work
 * units (image, pixel tile) are taken from an atomic queue in descending
 * emitter count.
 *
 * Replaces the reference kernels wfkernelf / wfkerneld
 * (idi/simulation/sim.cu:141-149) and their per-image launch loop in
 * idi/simulation/cuda.py:88-136; IDIWF_DOUBLE follows the FP64 CPU kernel
 * idi/simulation/cpu.py:68-107.  Amplitudes (per-emitter a_j) and batching
 * have no reference counterpart.
 *
 * IDIWF_SPLIT in the near field (IDIWF_NF) picks a path per image from the
 * image's largest |r| and the detector plane's distance D from the origin:
 * the second-order path difference where the dropped remainder is below
 * 1e-7 rad (and, with IDIWF_SCALE, (|r|/D)^2 <= 1e-7), else an exact
 * per-pair remainder at about half the speed.  Images with |r| > D/4 or a
 * remainder above 2 rad are not computed: the call records
 * IDIWF_ERR_UNSUPPORTED in the workspace (idiwf_workspace_error); the FP64
 * kernel (IDIWF_DOUBLE) has no such limit.
 */
idiwf_status idiwf_forward(const idiwf_geom *geom, const idiwf_batch *batch, int32_t precision,
                           int32_t out_kind, void *out, void *workspace, size_t workspace_bytes,
                           const idiwf_config *cfg, cudaStream_t stream);

/* Per-CTA busy time of the last forward launch that used `workspace`
 * (nanoseconds, DEVICE->host copy + stream sync).  Fills up to `cap` entries,
 * returns the count in *n.  Used to report load imbalance. */
idiwf_status idiwf_forward_cta_times(const void *workspace, uint64_t *host_ns, int32_t cap,
                                     int32_t *n, cudaStream_t stream);

/*
 * Split-precision forward that allocates nothing: no device memory, no
 * workspace argument, no host heap.  It has no counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc or hand the library a workspace
 * (code running inside another framework's memory pool or allocator hooks,
 * or plug-ins whose host forbids device allocation).  Its scratch is a
 * static device array of IDIWF_NOALLOC_SCRATCH_BYTES (16 MiB) that every
 * GPU which loads this library holds until the process exits.
 *
 * Limits: at most 512 images per call, and the emitters of all images, each
 * image padded to a multiple of 256, must fit the scratch at 52 bytes each:
 * 321,792 emitters in total.  Larger batches are rejected with
 * IDIWF_ERR_UNSUPPORTED before anything is enqueued.
 *
 * The first call on a device looks up the array's device address (with that
 * device current); make that first call before any stream capture.  The
 * address is kept for the life of the process: after cudaDeviceReset the
 * library's module is loaded again elsewhere, so a process that resets a
 * device must not call this entry point on it afterwards.  All calls share
 * the one array and it keeps the last call's contents; each call clears what
 * must start at zero.  Calls whose work overlaps on the GPU (other streams,
 * other threads, other graph branches) race on the scratch: serialise them.
 *
 * Same kernels and paths as idiwf_forward with precision IDIWF_SPLIT and its
 * default shape; results agree with idiwf_forward to the split tolerance,
 * not bit for bit, because idiwf_forward splits small detectors over
 * emitter chunks (another summation order).  Device-side errors (emitter
 * coordinates out of range, a near-field image outside the split range, a
 * bounded wait that ran out) are read back with idiwf_forward_noalloc_error.
 */
#define IDIWF_NOALLOC_SCRATCH_BYTES (16u << 20)
idiwf_status idiwf_forward_noalloc(const idiwf_geom *geom, const idiwf_batch *batch, int32_t out_kind,
                                   void *out, cudaStream_t stream);

/* Device error word of the most recent idiwf_forward_noalloc call on the
 * current device, with the statuses of idiwf_workspace_error.  Allocates
 * nothing (the word is copied into a stack variable) and synchronises
 * `stream`.  No counterpart in the reference. */
idiwf_status idiwf_forward_noalloc_error(cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* adjoint                                                                   */
/* ------------------------------------------------------------------------ */

size_t idiwf_backward_workspace_size(const idiwf_geom *geom, const idiwf_batch *batch,
                                     const idiwf_config *cfg);

/*
 * Adjoint direct sum (split precision) of I = |E|^2: given the forward field
 * `field` (complex128, (n_images, nx, ny), from idiwf_forward) and the
 * upstream gradient `grad_intensity` = dL/dI ((n_images, nx, ny) float64),
 * writes
 *   grad_atoms (offsets[n], 4) float64: dL/dx, dL/dy, dL/dz, dL/dphase
 *   grad_amp   (offsets[n])    float64: dL/da (may be NULL)
 * No reference counterpart (the reference has no gradients).
 */
idiwf_status idiwf_backward(const idiwf_geom *geom, const idiwf_batch *batch,
                            const void *field, const double *grad_intensity, double *grad_atoms,
                            double *grad_amp, void *workspace, size_t workspace_bytes,
                            const idiwf_config *cfg, cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* time-dependent path                                                       */
/* ------------------------------------------------------------------------ */

/* Largest emitter count the on-chip per-pixel sort handles.  Above it (up to
 * 2^28 emitters) a kernel with the per-pixel keys and permutations in the
 * workspace runs instead, and the workspace grows with n. */
int64_t idiwf_time_max_emitters(void);

/* Workspace for n emitters on this detector (for n above
 * idiwf_time_max_emitters(): 32 n bytes per resident CTA on the current device). */
size_t idiwf_time_workspace_size(const idiwf_geom *geom, int64_t n);

/*
 * Time-dependent intensity (FP64): per pixel, arrival times t_j + path/c,
 * an on-chip sort by arrival time, the decaying coherent scan and the
 * analytic interval integral; out is (nx, ny) float64.
 * geom->offset must be zero (the reference time path has no detector offset).
 * Replaces simulated / simulatef / simulatedf and tempsize*
 * (idi/simulation/simtime.cu:170-278) driven by idi/simulation/cutime.py:9-139,
 * with the FP64 CPU semantics of idi/simulation/time.py:48-98.
 */
idiwf_status idiwf_time_forward(const idiwf_geom *geom, const double *atoms, const double *times,
                                int64_t n, double c, double tau, double *out, void *workspace,
                                size_t workspace_bytes, cudaStream_t stream);

/*
 * idiwf_time_forward plus, for every pixel, a 64-bit digest of its sorted
 * emitter order, digest[p] = sum_m (j_m + 1) B^m mod 2^64 over the emitter
 * indices j_m in arrival order, B = 0x9E3779B97F4A7C15 (a swap of any two
 * emitters changes it).  digest is DEVICE (nx, ny) uint64.  Verification
 * helper: it lets a caller compare every pixel's order with another sort of
 * the same keys without storing n indices per pixel.  No counterpart in the
 * reference.
 */
idiwf_status idiwf_time_forward_digest(const idiwf_geom *geom, const double *atoms, const double *times,
                                       int64_t n, double c, double tau, double *out, uint64_t *digest,
                                       void *workspace, size_t workspace_bytes, cudaStream_t stream);

/*
 * Sorted emitter order of one pixel, as the time path computes it
 * (order[m] = emitter of the m-th earliest arrival; sorted_keys[m] its
 * arrival time).  Verification helper for bit-exact ordering; device outputs.
 * Mirrors the argsort of idi/simulation/time.py:19-29.
 */
idiwf_status idiwf_time_order(const idiwf_geom *geom, const double *atoms, const double *times,
                              int64_t n, double c, int32_t ix, int32_t iy, int32_t *order,
                              double *sorted_keys, void *workspace, size_t workspace_bytes,
                              cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* detector: photon sampling and charge sharing                              */
/* ------------------------------------------------------------------------ */

/*
 * Counter-based random stream: Philox4x64-10 (Salmon, Moraes, Dror, Shaw,
 * "Parallel random numbers: as easy as 1, 2, 3", SC 2011) with the counter
 * convention of numpy.random.Philox: a stream with counter (0, c1, c2, c3)
 * yields the blocks of counters (1, c1, c2, c3), (2, c1, c2, c3), ..., four
 * 64-bit words each, and a uniform double is (word >> 11) * 2^-53.  So
 * numpy.random.Generator(numpy.random.Philox(counter=[0, c1, c2, c3],
 * key=key)).random() reproduces a stream bit for bit.  `stream` is counter
 * word 3: calls that should draw independent numbers use distinct values.
 */
typedef struct idiwf_rng {
    uint64_t key[2];
    uint64_t stream;
    uint64_t first_image; /* image b of a call draws as image first_image + b, so a
                             batch split over several calls draws the same numbers */
} idiwf_rng;

/* Bytes of workspace idiwf_photons needs. */
size_t idiwf_photons_workspace_size(int32_t n_images, int64_t npix);

/*
 * Poisson photon counts on the device:
 *     out[b, p] ~ Poisson(probs[b, p] * (n_photons / sum_p probs[b, p]))
 * for every image b of `probs` ((n_images, npix), DEVICE, probs_dtype
 * IDIWF_F64 or IDIWF_F32; the rate is formed in FP64).  out_dtype: IDIWF_F64,
 * IDIWF_F32, IDIWF_I32, IDIWF_U32 or IDIWF_I64 (the reference's `dtype`).
 *
 * Replaces idi/simulation/common.py:11-23 randomphotons, which calls
 * numpy's / cupy's Generator.poisson on the host or device array.  The
 * per-image sum is a fixed-order FP64 reduction (deterministic; within a few
 * ulps of numpy's pairwise sum).  Pixel p of image b draws from its own
 * stream, counter (0, p, rng->first_image + b, rng->stream), so results do
 * not depend on the launch shape or on how a batch is split into calls.  Sampler: inversion by sequential search for rates below 10,
 * otherwise the transformed rejection with squeeze PTRS (W. Hoermann, "The
 * transformed rejection method for generating Poisson random variables",
 * Insurance: Mathematics and Economics 12, 1993).  A negative or NaN
 * probability or an all-zero image records an invalid-value error in the
 * workspace (idiwf_workspace_error) and yields zero counts for the pixel.
 * n_photons must be finite and >= 0 (the reference returns `probs`
 * unchanged for infinite n_photons; the host side handles that case).
 */
idiwf_status idiwf_photons(const void *probs, int32_t probs_dtype, int32_t n_images, int64_t npix,
                           double n_photons, const idiwf_rng *rng, void *out, int32_t out_dtype,
                           void *workspace, size_t workspace_bytes, cudaStream_t stream);

/* Bytes of workspace idiwf_chargesharing needs (`injected`: nonzero when
 * `positions` will be given). */
size_t idiwf_chargesharing_workspace_size(int32_t n_images, int32_t nx, int32_t ny, int32_t injected);

/*
 * Charge sharing between neighbouring pixels (idi/simulation/common.py:26-67):
 * every photon counted in pixel (ix, iy) of `counts` ((n_images, nx, ny),
 * DEVICE, counts_dtype IDIWF_F64/F32/I32/U32/I64, truncated toward zero as
 * numpy's astype(int)) lands at offset mu = (mu_x, mu_y) in [-0.5, 0.5)^2
 * from the pixel centre and deposits into pixel (ix + dr, iy + dc),
 * |dr|, |dc| <= w = ceil(2 s), the charge
 *     1/4 [erf(c + a_x) + erf(c - a_x)] [erf(c + a_y) + erf(c - a_y)],
 *     a_x = (mu_x - dc) / (sqrt(2) s),  a_y = (mu_y - dr) / (sqrt(2) s),
 *     c = 1 / (2 sqrt(2) s),
 * times its scale (1 when ns == 0); charge leaving the detector is lost.
 * The pairing of mu_x with the column offset follows the reference's
 * deposit loop (common.py:63-67).  For s <= 0 the result is
 * counts * scale per pixel (counts itself when ns == 0), as in common.py:35-39.
 * out: DEVICE (n_images, nx, ny) float64.  Each output pixel gathers its
 * neighbours' photons in the reference's photon order, so every pixel sums
 * in the same order as the reference's scatter loop (deterministic).
 *
 * Random draws, generated mode (positions == NULL): photon i of pixel p of
 * image b uses the first block of the stream with counter
 * (i, p, (rng->first_image + b) | 2^63, rng->stream): words 0 and 1 give mu_x, mu_y (uniform
 * - 0.5), words 2 and 3 a Box-Muller normal z; scale = 1 + ns z.  For
 * s <= 0, pixel p uses counter (0, p, (rng->first_image + b) | 2^62,
 * rng->stream) the same way.
 * Injected mode: `positions` (n_positions, 2) float64 mu of every photon and
 * `scales` (n_positions) float64 factors or NULL, in the reference's photon
 * order (image, then row-major pixel, then photon within the pixel); for
 * s <= 0, `scales` holds one factor per pixel.  A photon total different
 * from n_positions records an invalid-value error in the workspace.
 */
idiwf_status idiwf_chargesharing(const void *counts, int32_t counts_dtype, int32_t n_images, int32_t nx,
                                 int32_t ny, double s, double ns, const idiwf_rng *rng,
                                 const double *positions, const double *scales, int64_t n_positions,
                                 double *out, void *workspace, size_t workspace_bytes, cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* emitter sources on the device                                             */
/* ------------------------------------------------------------------------ */

/* emitter families (the reference's simulation objects, idi/simulation/simobj.py) */
#define IDIWF_EMIT_SPHERE 0 /* uniform in a ball of radius r: rndSphere (idi/util/random.py:39-51), simobj.py:119-130 */
#define IDIWF_EMIT_GNORM 1  /* generalised normal volume: gnorm / gauss (simobj.py:154-184,
                               rndgennorm idi/util/random.py:6-26) */
#define IDIWF_EMIT_FOIL 2   /* foil: in-plane generalised normal, depth uniform or truncated
                               exponential (simobj.py:703-760, rndtruncexp idi/util/random.py:142-151) */
#define IDIWF_EMIT_SITES 3  /* subsample of lattice sites without replacement, optionally
                               weighted and randomly oriented: crystal.updatePos (simobj.py:446-487) */
#define IDIWF_EMIT_FIXED 4  /* the same positions in every image (rndPos = False), new phases */

/* SITES orientation per image */
#define IDIWF_ORIENT_FIXED 0   /* positions = rot @ site */
#define IDIWF_ORIENT_RANDOM 1  /* uniformly random rotation A per image (idi/util/random.py:130-139):
                                  positions = A @ rot @ site */
#define IDIWF_ORIENT_AXIS 2    /* random angle about `axis` (idi/util/__init__.py:338-345) */

typedef struct idiwf_emitters_desc {
    int32_t kind;         /* IDIWF_EMIT_* */
    int32_t random_phase; /* nonzero: phase ~ U[0, 2 pi) per emitter and image (rndPhase); zero: 0 */
    int32_t orientation;  /* SITES: IDIWF_ORIENT_* */
    int32_t weighted;     /* SITES: weight site i by exp(-sum_a |x_a|^rho_a ln2 (2/fwhm_a)^rho_a)
                             of its rotated position (the crystal's fwhm envelope) */
    double r;             /* SPHERE: radius */
    double fwhm[3];       /* GNORM: per axis; FOIL: [0], [1] in plane; SITES: envelope */
    double rho[3];        /* shape (2 = Gaussian) of the same */
    double depth;         /* FOIL: path through the foil, thickness / rot[8] */
    double attenuation;   /* FOIL: attenuation length; not finite or <= 0: uniform depth */
    double rot[9];        /* GNORM, FOIL, SITES, FIXED: row-major rotation applied to positions */
    double axis[3];       /* SITES with IDIWF_ORIENT_AXIS */
    const double *sites;  /* SITES, FIXED: DEVICE (n_sites, 3) float64 */
    int64_t n_sites;      /* SITES: lattice sites; FIXED: must equal n */
} idiwf_emitters_desc;

size_t idiwf_emitters_workspace_size(const idiwf_emitters_desc *desc, int32_t n_images, int64_t n);

/*
 * Emitters of n_images images, n each, generated on the device into `atoms`
 * (DEVICE, (n_images * n, 4) float64 [x, y, z, phase], the forward's input
 * layout), replacing the host simobject.get2() draws that feed
 * idi/simulation/cuda.py:89,115.  Emitter j of image b draws from the stream
 * with counter (0, j, (rng->first_image + b) | 2^61, rng->stream): so a batch
 * split into several calls (first_image) draws the same emitters.  The
 * numbers differ from the reference's numpy draws; the distributions are the
 * reference's.
 *   SPHERE: t = 2u0 - 1, p = 2 pi u1, radius r cbrt(u2), phase 2 pi u3.
 *   GNORM:  rho == 2 on every axis: x_a = N(0,1) fwhm_a / 2.355 (Box-Muller);
 *           otherwise x_a = +-fwhm_a/2 (G_a / ln 2)^(1/rho_a), G_a ~
 *           Gamma(1/rho_a) (G. Marsaglia, W. Tsang, ACM TOMS 26, 2000).  Then rot.
 *   FOIL:   in plane as GNORM with fwhm / 2.35 (the reference's constant for
 *           foils), mapped by rot's first two columns; z += depth draw:
 *           -lam log1p(u expm1(-depth/lam)) or u depth.
 *   SITES:  per image and round (n > n_sites takes ceil(n / n_sites) rounds of
 *           at most n_sites distinct sites, as the reference's repeated
 *           choice), the smallest keys -log(1-u_i)/w_i (weighted; u_i
 *           otherwise) -- the successive weighted sampling without replacement
 *           of numpy's choice(replace=False, p=w/sum w), by the exponential-key
 *           method of P. Efraimidis, P. Spirakis (Inf. Proc. Letters 97, 2006)
 *           -- selected by an exact radix select (ties by site index) and
 *           written in site order.  Fewer positive weights than needed records
 *           an invalid-value error.
 *   FIXED:  sites[j] every image.
 */
idiwf_status idiwf_emitters(const idiwf_emitters_desc *desc, int32_t n_images, int64_t n, const idiwf_rng *rng,
                            double *atoms, void *workspace, size_t workspace_bytes, cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* direct q-space autocorrelation of detector images                         */
/* ------------------------------------------------------------------------ */

/*
 * Both correlators sum v(p) v(p') over pixel pairs p = (r, c), p' = (r + dr,
 * c + dc) with 0 <= dr < qmax and |dc| <= qmax (radial) or < qmax (3d), the
 * pair set of the reference's launch grids, and bin each pair by the
 * difference of the pixels' q vectors.  Each thread walks one column offset
 * along a row pair and sums the products of consecutive pairs that fall in
 * the same bin in FP32 before adding the run to the FP64 histogram (the
 * radial reference kernel does the same; the 3d one adds every pair to FP32
 * bins, which agree with these sums to FP32 rounding).  Images are
 * (n_images, nr, nc) float32, DEVICE.  Results are deterministic up to the
 * order of FP64 additions.
 */
size_t idiwf_qcorr_workspace_size(int32_t nr, int32_t nc);

/*
 * Radial correlation, idi/reconstruction/cucorrad.py:10-152: bin
 * round(|q(p) - q(p')|) (FP32, round half to even), bins 0..qmax-1 into out
 * (n_images, qmax) float64.  q: DEVICE (nr * nc, 4) float32 rows
 * [qx, qy, qz, unused] (the reference's float32 q = k z / d), 16-byte
 * aligned; nc <= 4096, qmax <= 511.  As in the reference, a run is added when
 * the bin changes, and at the end of a row pair only if the last pair's bin
 * is below qmax (cucorrad.py:102-116).
 */
idiwf_status idiwf_qcorr_radial(const float *q, const float *images, int32_t n_images, int32_t nr, int32_t nc,
                                int32_t qmax, double *out, void *workspace, size_t workspace_bytes,
                                cudaStream_t stream);

/*
 * 3d correlation, idi/reconstruction/cucor.py:10-128: bin
 *   (maxdqz + round(z (zd(p) - zd(p'))),
 *    qmax + round((c' - yc) zd(p') - (c - yc) zd(p)),
 *    qmax + round((r' - xc) zd(p') - (r - xc) zd(p)))
 * (FP32, round half to even) into out (n_images, 2 maxdqz, 2 qmax, 2 qmax)
 * float64, then symmetrise it about the centre as the reference's assemble
 * step does (cucor.py:101-104, x extent of its launch): bins i and -i (mod
 * the shape) both receive the sum of the two, a bin that is its own mirror
 * doubles.  zd: DEVICE (nr, nc) float32 z / d; nc <= 8192, qmax <= 1024.
 * Pairs whose bin falls outside the array are dropped (the reference's kernel
 * writes them past the end of its array).
 */
idiwf_status idiwf_qcorr_3d(const float *zd, const float *images, int32_t n_images, int32_t nr, int32_t nc,
                            int32_t qmax, int32_t maxdqz, float xcenter, float ycenter, float z, double *out,
                            void *workspace, size_t workspace_bytes, cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* FFT autocorrelation                                                      */
/* ------------------------------------------------------------------------ */

/*
 * The whole autocorrelation of idi/reconstruction/cusimple.py:6-38 along two
 * axes, by this library's own FFTs: for each of `batch` images x[b] (n0 x n1
 * of dtype, row-major, contiguous, batch-major),
 *     out[b] = crop(fftshift(irfft2(|rfft2(x[b], (G0, G1))|^2)))
 * ((2 n0) x (2 n1) of dtype; for powers of two G = 2 n and the crop is the
 * whole shifted array).  Then,
 * per output position (i, j): mode -1 nothing; mode 0 y / norm, NaN where
 * norm < threshold; mode 1 y / norm where norm > threshold, else 0 (norm:
 * (2 n0) x (2 n1) of dtype); mode 2 y / count with the pair count
 * count = (n0 - |i - n0|)(n1 - |j - n1|), NaN where count < threshold (the
 * norm=True result of cusimple.py:23-34 without a second transform).
 * Shapes: n0, n1 powers of two from 4 to 4096 (x and out aligned to two
 * elements), or any n0, n1 >= 1 whose padded lengths G0 = fastlen(2 n0) and
 * G1 = fastlen(2 n1) (smallest products of 2, 3, 5, 7, 11, as
 * idi.util.fastlen) are at most 4096; out is then the centre crop
 * (i - n0) mod G0, (j - n1) mod L1 of the shifted array, as the reference's
 * slice, with L1 = G1 for an even G1 and G1 - 1 for an odd one (numpy's
 * default inverse length; mode 2 is then IDIWF_ERR_UNSUPPORTED, since the
 * reference's pair count is the same transform of ones: pass it as norm with
 * mode 0).  Other shapes: IDIWF_ERR_UNSUPPORTED.
 * workspace: idiwf_fft_autocorr_workspace_size() bytes for this batch and
 * shape, 256-byte aligned (twiddle tables and the intermediates of one group
 * of images; groups run one after another; 0 for unsupported arguments).
 */
size_t idiwf_fft_autocorr_workspace_size(int64_t batch, int32_t n0, int32_t n1, int32_t dtype);
idiwf_status idiwf_fft_autocorr(const void *x, int32_t dtype, int64_t batch, int32_t n0, int32_t n1,
                                const void *norm, int32_t mode, double threshold, void *out, void *workspace,
                                size_t workspace_bytes, cudaStream_t stream);

/*
 * The autocorrelation of each of `lines` independent lines (x: lines x n of
 * dtype, contiguous) along its length, as cusimple.py:6-38 with one
 * correlated axis: out (lines x 2n) = crop(fftshift(irfft(|rfft(x, G)|^2)))
 * with G = fastlen(2 n) at most 4096 (else IDIWF_ERR_UNSUPPORTED; an odd G
 * as for idiwf_fft_autocorr).  Modes as idiwf_fft_autocorr, with the pair count
 * n - |j - n| and norm of 2n values.  workspace:
 * idiwf_fft_autocorr_1d_workspace_size() bytes, 256-byte aligned.
 */
size_t idiwf_fft_autocorr_1d_workspace_size(int64_t lines, int32_t n, int32_t dtype);
idiwf_status idiwf_fft_autocorr_1d(const void *x, int32_t dtype, int64_t lines, int32_t n, const void *norm,
                                   int32_t mode, double threshold, void *out, void *workspace,
                                   size_t workspace_bytes, cudaStream_t stream);

/* Helpers around a library FFT (other shapes). */

/* In place |X|^2 of n complex values (dtype IDIWF_F64: complex128, IDIWF_F32:
 * complex64): re <- re^2 + im^2, im <- 0.  The `ret = abs(ret) ** 2` of
 * idi/reconstruction/cusimple.py:20 and :70. */
idiwf_status idiwf_power_spectrum(void *spectrum, int64_t n, int32_t dtype, cudaStream_t stream);

/*
 * Centre crop of an inverse-transformed autocorrelation, fused with its
 * normalisation: for every batch entry b and index i (up to 3 trailing axes),
 *     y = full[b, (i_k - n_k) mod g_k ...]      (fftshift, then the
 *                                                 [F/2 - n, F/2 + n) slice)
 * full: (batch, g...) of dtype, out: (batch, 2n...) of dtype.  With `norm`
 * ((2n...) of dtype): mode 0 gives y / norm, NaN where norm < threshold
 * (cusimple.py:23-34); mode 1 gives y / norm where norm > threshold, else 0
 * (the correlator's division, cusimple.py:38).  Without norm, y.
 * Replaces the fftshift / slice / divide steps of cusimple.py:22-34,72-95.
 */
idiwf_status idiwf_corr_crop(const void *full, int32_t dtype, int64_t batch, int32_t ndim, const int32_t *g,
                             const int32_t *n, const void *norm, int32_t mode, double threshold, void *out,
                             cudaStream_t stream);

/*
 * The running mean / variance update of idi/reconstruction/cusimple.py:97-105
 * (Welford), FP32 like the reference: with count the number of samples after
 * adding x, count == 1 sets mean = x, nvar = 0; otherwise
 * delta = x - mean, mean += delta / count, nvar += delta (x - mean).
 */
idiwf_status idiwf_welford_update(const float *x, float *mean, float *nvar, int64_t n, int64_t count,
                                  cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* tuning, diagnostics                                                       */
/* ------------------------------------------------------------------------ */

/*
 * Autotune the forward kernel shape for this geometry/batch/precision: times
 * each candidate idiwf_config on a subsample of the work with CUDA events and
 * caches the fastest under a key of (precision, flags, nx, ny, emitter-count
 * bucket).  Later idiwf_forward calls with cfg == NULL use the cached shape.
 * Synchronises `stream`.  Writes the chosen shape to *best when non-NULL.
 */
idiwf_status idiwf_tune(const idiwf_geom *geom, const idiwf_batch *batch, int32_t precision,
                        int32_t out_kind, void *out, void *workspace, size_t workspace_bytes,
                        cudaStream_t stream, idiwf_config *best);

/* Reads the device error word of `workspace` (synchronises `stream`): the
 * errors of the most recent call that used this workspace (every call clears
 * the word when it starts).  Returns IDIWF_OK, IDIWF_ERR_TIMEOUT when a
 * bounded wait gave up, or IDIWF_ERR_UNSUPPORTED when emitter coordinates
 * were outside the split-precision phase range. */
idiwf_status idiwf_workspace_error(const void *workspace, cudaStream_t stream);

/*
 * Pipe-throughput microbenchmark used to measure the roofline denominators:
 * kind 0 = MUFU sin+cos (ops/s), 1 = FP64 FMA (flop/s counted as 2 per FMA),
 * 2 = FP32 FMA, 3 = packed FP32x2 FMA.  Runs on `stream`, synchronises it and
 * returns the measured rate in *rate.  scratch: DEVICE, >= 4 MiB.
 */
idiwf_status idiwf_microbench(int32_t kind, void *scratch, cudaStream_t stream, double *rate);

/* Human-readable description of the last error on the calling thread. */
const char *idiwf_last_error_string(void);

/* Library version, ABI version in the high 16 bits. */
int32_t idiwf_version(void);

#ifdef __cplusplus
}
#endif
#endif /* IDIWF_H */
