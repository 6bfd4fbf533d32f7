// Emitter sources on the device: the reference's simulation objects
// (idi/simulation/simobj.py) drawn straight into the forward's (n, 4)
// [x, y, z, phase] rows in HBM.
//
//  * emit_kernel<KIND> — SPHERE, GNORM, FOIL, FIXED: one thread per emitter,
//    draws from the emitter's own Philox stream (counter (0, j, img | 2^61,
//    stream)).
//  * sites_rot_kernel — per image, the rotation applied to the lattice sites
//    (random per image: stream counter (0, 2^64 - 1, img | 2^61, stream)).
//  * sites_key_kernel — per site, the exponential key of weighted sampling
//    without replacement (stream counter (0, i, img | 2^60 | round << 44,
//    stream)), stored as the bits of a non-negative double (monotone as
//    unsigned integers).
//  * sites_select_kernel — one CTA per image: 8 passes of an 8-bit radix
//    select find the k-th smallest key exactly, then a block scan writes the
//    selected sites (key below the threshold, or equal to it in site order up
//    to the count) in site order.
#include <cmath>

#include "idiwf_internal.cuh"
#include "philox.cuh"

namespace idiwf {

constexpr uint64_t kEmitTag = 1ull << 61;
constexpr uint64_t kSiteTag = 1ull << 60;
constexpr int kRoundShift = 44;
constexpr double kLn2 = 0.69314718055994530942;

struct EmitParams {
    int32_t kind, random_phase, orientation, weighted;
    double r;
    double fwhm[3], rho[3];
    double s[3];  // ln2 (2 / fwhm)^rho: envelope coefficients (SITES)
    double depth, attenuation;
    double rot[9];
    double axis[3];
    const double *sites;
    int64_t n_sites;
    int64_t n;
    uint64_t k0, k1, stream, img0;
};

__device__ __forceinline__ double normal(PhiloxStream &st) {
    const double a = st.uniform();
    const double b = st.uniform();
    return box_muller(a, b);
}

// Gamma(a, 1), a > 0: G. Marsaglia, W. Tsang, "A simple method for generating
// gamma variables", ACM TOMS 26 (2000); a < 1 through G(a+1) U^(1/a).
// Returns -1 when the (bounded) rejection loop ran out.
__device__ double gamma_draw(double a, PhiloxStream &st) {
    double boost = 1.0;
    if (a < 1.0) {
        boost = pow(1.0 - st.uniform(), 1.0 / a);
        a += 1.0;
    }
    const double d = a - 1.0 / 3.0;
    const double c = 1.0 / sqrt(9.0 * d);
    for (int trial = 0; trial < 1000; ++trial) {
        double x, v;
        int inner = 0;
        do {
            x = normal(st);
            v = 1.0 + c * x;
        } while (v <= 0.0 && ++inner < 1000);
        v = v * v * v;
        const double u = 1.0 - st.uniform();
        const double x2 = x * x;
        if (u < 1.0 - 0.0331 * x2 * x2) return d * v * boost;
        if (log(u) < 0.5 * x2 + d * (1.0 - v + log(v))) return d * v * boost;
    }
    return -1.0;
}

// one generalised-normal coordinate with full width at half maximum `fwhm`
// (idi/util/random.py:6-26): +-fwhm/2 (G / ln 2)^(1/rho), G ~ Gamma(1/rho)
__device__ __forceinline__ double gennorm_draw(double fwhm, double rho, PhiloxStream &st, bool &bad) {
    const double sign = st.uniform() < 0.5 ? -1.0 : 1.0;
    const double g = gamma_draw(1.0 / rho, st);
    if (g < 0.0) bad = true;
    return fwhm * 0.5 * pow(fmax(g, 0.0) / kLn2, 1.0 / rho) * sign;
}

__device__ __forceinline__ void rotate(const double *M, double x, double y, double z, double &ox, double &oy,
                                       double &oz) {
    ox = M[0] * x + M[1] * y + M[2] * z;
    oy = M[3] * x + M[4] * y + M[5] * z;
    oz = M[6] * x + M[7] * y + M[8] * z;
}

template <int KIND>
__global__ void __launch_bounds__(256) emit_kernel(const EmitParams P, double *__restrict__ atoms,
                                                   uint32_t *__restrict__ err) {
    const int b = blockIdx.y;
    const uint64_t img = P.img0 + (uint64_t)b;
    bool bad = false;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < P.n; j += (int64_t)gridDim.x * blockDim.x) {
        PhiloxStream st((uint64_t)j, img | kEmitTag, P.stream, P.k0, P.k1);
        double x, y, z;
        if (KIND == IDIWF_EMIT_SPHERE) {
            const double t = 2.0 * st.uniform() - 1.0;
            const double p2 = 2.0 * st.uniform();  // azimuth in units of pi
            const double u = P.r * cbrt(st.uniform());
            const double s = sqrt(1.0 - t * t);
            double sp, cp;
            sincospi(p2, &sp, &cp);
            x = u * t;
            y = u * s * sp;
            z = u * s * cp;
        } else if (KIND == IDIWF_EMIT_GNORM) {
            double v[3];
            if (P.rho[0] == 2.0 && P.rho[1] == 2.0 && P.rho[2] == 2.0) {
                double z3;
                box_muller2(st.uniform(), st.uniform(), v[0], v[1]);
                box_muller2(st.uniform(), st.uniform(), v[2], z3);
#pragma unroll
                for (int a = 0; a < 3; ++a) v[a] *= P.fwhm[a] / 2.355;
            } else {
#pragma unroll
                for (int a = 0; a < 3; ++a) v[a] = gennorm_draw(P.fwhm[a], P.rho[a], st, bad);
            }
            rotate(P.rot, v[0], v[1], v[2], x, y, z);
        } else if (KIND == IDIWF_EMIT_FOIL) {
            double v0, v1;
            if (P.rho[0] == 2.0 && P.rho[1] == 2.0) {
                box_muller2(st.uniform(), st.uniform(), v0, v1);
                v0 *= P.fwhm[0] / 2.35;
                v1 *= P.fwhm[1] / 2.35;
            } else {
                v0 = gennorm_draw(P.fwhm[0], P.rho[0], st, bad);
                v1 = gennorm_draw(P.fwhm[1], P.rho[1], st, bad);
            }
            x = P.rot[0] * v0 + P.rot[1] * v1;
            y = P.rot[3] * v0 + P.rot[4] * v1;
            z = P.rot[6] * v0 + P.rot[7] * v1;
            const double u = st.uniform();
            if (P.attenuation > 0.0 && isfinite(P.attenuation))
                z += -log1p(u * expm1(-P.depth / P.attenuation)) * P.attenuation;
            else
                z += u * P.depth;
        } else {  // FIXED
            const double *s = P.sites + 3 * j;
            rotate(P.rot, s[0], s[1], s[2], x, y, z);
        }
        const double phase = P.random_phase ? 2.0 * M_PI * st.uniform() : 0.0;
        double *row = atoms + ((int64_t)b * P.n + j) * 4;
        reinterpret_cast<double2 *>(row)[0] = make_double2(x, y);
        reinterpret_cast<double2 *>(row)[1] = make_double2(z, phase);
    }
    if (bad) record_error(err, kErrValue);
}

// ---------------------------------------------------------------------------
// lattice-site subsampling
// ---------------------------------------------------------------------------
// rotation of image b's sites: fixed rot, or A @ rot with A random
__global__ void sites_rot_kernel(const EmitParams P, int n_images, double *__restrict__ rots) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n_images) return;
    double A[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    if (P.orientation != IDIWF_ORIENT_FIXED) {
        PhiloxStream st(~0ull, (P.img0 + (uint64_t)b) | kEmitTag, P.stream, P.k0, P.k1);
        if (P.orientation == IDIWF_ORIENT_RANDOM) {
            // J. Arvo, "Fast random rotation matrices", Graphics Gems III (1992):
            // a rotation about z by theta, then the reflection 2 V V^T - I
            const double th2 = 2.0 * st.uniform(), ph2 = 2.0 * st.uniform(), zz = st.uniform();
            double sp, cp, st_, ct;
            sincospi(ph2, &sp, &cp);
            sincospi(th2, &st_, &ct);
            const double V[3] = {cp * sqrt(zz), sp * sqrt(zz), sqrt(1.0 - zz)};
            const double R[9] = {ct, st_, 0.0, -st_, ct, 0.0, 0.0, 0.0, 1.0};
            double H[9];
            for (int i = 0; i < 3; ++i)
                for (int k = 0; k < 3; ++k) H[3 * i + k] = 2.0 * V[i] * V[k] - (i == k ? 1.0 : 0.0);
            for (int i = 0; i < 3; ++i)
                for (int k = 0; k < 3; ++k) A[3 * i + k] = H[3 * i] * R[k] + H[3 * i + 1] * R[3 + k] + H[3 * i + 2] * R[6 + k];
        } else {
            // Rodrigues: cos t I + sin t [u]_x + (1 - cos t) u u^T, t ~ U[0, 2 pi)
            const double nrm = sqrt(P.axis[0] * P.axis[0] + P.axis[1] * P.axis[1] + P.axis[2] * P.axis[2]);
            const double u[3] = {P.axis[0] / nrm, P.axis[1] / nrm, P.axis[2] / nrm};
            double s, c;
            sincospi(2.0 * st.uniform(), &s, &c);
            const double K[9] = {0.0, -u[2], u[1], u[2], 0.0, -u[0], -u[1], u[0], 0.0};
            for (int i = 0; i < 3; ++i)
                for (int k = 0; k < 3; ++k) A[3 * i + k] = (i == k ? c : 0.0) + s * K[3 * i + k] + (1.0 - c) * u[i] * u[k];
        }
    }
    double *M = rots + 9 * (int64_t)b;
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) M[3 * i + k] = A[3 * i] * P.rot[k] + A[3 * i + 1] * P.rot[3 + k] + A[3 * i + 2] * P.rot[6 + k];
}

__global__ void __launch_bounds__(256) sites_key_kernel(const EmitParams P, int round, const double *__restrict__ rots,
                                                        uint64_t *__restrict__ keys) {
    const int b = blockIdx.y;
    const double *M = rots + 9 * (int64_t)b;
    const uint64_t tag = (P.img0 + (uint64_t)b) | kSiteTag | ((uint64_t)round << kRoundShift);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P.n_sites;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t w0, w1, w2, w3;
        philox4x64(1, (uint64_t)i, tag, P.stream, P.k0, P.k1, w0, w1, w2, w3);
        const double u = u01(w0);
        double key = u;
        if (P.weighted) {
            const double *s = P.sites + 3 * i;
            double x[3];
            rotate(M, s[0], s[1], s[2], x[0], x[1], x[2]);
            double e = 0.0;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const double ax = fabs(x[a]);
                e += (P.rho[a] == 2.0 ? ax * ax : pow(ax, P.rho[a])) * P.s[a];
            }
            const double w = exp(-e);
            key = w > 0.0 ? -log1p(-u) / w : INFINITY;
        }
        keys[(int64_t)b * P.n_sites + i] = (uint64_t)__double_as_longlong(key);
    }
}

constexpr int kSelThreads = 1024;

// exclusive scan over the CTA (kSelThreads threads); *total gets the sum
__device__ __forceinline__ uint32_t cta_exclusive_scan(uint32_t x, uint32_t *warp_sums, uint32_t *total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += y;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kSelThreads / 32 ? warp_sums[lane] : 0;
        uint32_t wi = w;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, wi, d);
            if (lane >= d) wi += y;
        }
        warp_sums[lane] = wi - w;  // exclusive per warp
        if (lane == 31) warp_sums[32] = wi;
    }
    __syncthreads();
    const uint32_t r = warp_sums[warp] + incl - x;
    *total = warp_sums[32];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kSelThreads) sites_select_kernel(const EmitParams P, int64_t take, int64_t base,
                                                                   const double *__restrict__ rots,
                                                                   const uint64_t *__restrict__ keys,
                                                                   double *__restrict__ atoms,
                                                                   uint32_t *__restrict__ err) {
    __shared__ uint32_t hist[256];
    __shared__ uint32_t warp_sums[33];
    __shared__ uint64_t s_prefix;
    __shared__ int64_t s_rem;
    const int b = blockIdx.x;
    const int64_t M = P.n_sites;
    const uint64_t *kb = keys + (int64_t)b * M;
    const double *R = rots + 9 * (int64_t)b;
    uint64_t prefix = 0, mask = 0;
    if (threadIdx.x == 0) s_rem = take;
    for (int shift = 56; shift >= 0; shift -= 8) {
        for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        for (int64_t i = threadIdx.x; i < M; i += blockDim.x) {
            const uint64_t k = kb[i];
            if ((k & mask) == prefix) atomicAdd(&hist[(k >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int64_t rem = s_rem, cum = 0;
            int digit = 255;
            for (int d = 0; d < 256; ++d) {
                if (cum + (int64_t)hist[d] >= rem) {
                    digit = d;
                    break;
                }
                cum += hist[d];
            }
            s_rem = rem - cum;
            s_prefix = prefix | ((uint64_t)digit << shift);
        }
        __syncthreads();
        prefix = s_prefix;
        mask |= 0xFFull << shift;
    }
    const uint64_t T = prefix;
    const int64_t n_eq = s_rem;  // keys equal to T to take, in site order
    if (threadIdx.x == 0 && __longlong_as_double((long long)T) == INFINITY) record_error(err, kErrValue);
    int64_t run_eq = 0, run_sel = 0;
    const uint64_t tag = (P.img0 + (uint64_t)b);
    for (int64_t c = 0; c < M; c += blockDim.x) {
        const int64_t i = c + threadIdx.x;
        const uint64_t k = i < M ? kb[i] : ~0ull;
        const bool less = i < M && k < T;
        const bool eq = i < M && k == T;
        uint32_t tot_eq, tot_sel;
        const uint32_t eq_rank = cta_exclusive_scan(eq ? 1u : 0u, warp_sums, &tot_eq);
        const bool sel = less || (eq && run_eq + (int64_t)eq_rank < n_eq);
        const uint32_t slot = cta_exclusive_scan(sel ? 1u : 0u, warp_sums, &tot_sel);
        if (sel) {
            const int64_t j = base + run_sel + slot;  // emitter index within the image
            if (j < P.n) {
                const double *s = P.sites + 3 * i;
                double x, y, z;
                rotate(R, s[0], s[1], s[2], x, y, z);
                double phase = 0.0;
                if (P.random_phase) {
                    PhiloxStream st((uint64_t)j, tag | kEmitTag, P.stream, P.k0, P.k1);
                    phase = 2.0 * M_PI * st.uniform();
                }
                double *row = atoms + ((int64_t)b * P.n + j) * 4;
                reinterpret_cast<double2 *>(row)[0] = make_double2(x, y);
                reinterpret_cast<double2 *>(row)[1] = make_double2(z, phase);
            }
        }
        run_eq += tot_eq;
        run_sel += tot_sel;
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static size_t emitters_ws_bytes(const idiwf_emitters_desc *d, int32_t n_images) {
    size_t bytes = 256 + align256((size_t)n_images * 9 * sizeof(double));
    if (d->kind == IDIWF_EMIT_SITES) bytes += align256((size_t)n_images * (size_t)d->n_sites * sizeof(uint64_t));
    return bytes;
}

static int emit_sms() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

}  // namespace idiwf

using namespace idiwf;

extern "C" size_t idiwf_emitters_workspace_size(const idiwf_emitters_desc *desc, int32_t n_images, int64_t n) {
    if (!desc || n_images <= 0 || n < 0) return 0;
    return emitters_ws_bytes(desc, n_images);
}

extern "C" idiwf_status idiwf_emitters(const idiwf_emitters_desc *desc, int32_t n_images, int64_t n,
                                       const idiwf_rng *rng, double *atoms, void *workspace, size_t workspace_bytes,
                                       cudaStream_t stream) {
    if (!desc || !rng) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "desc and rng must be non-NULL");
    if (n_images <= 0 || n_images > 65535) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "n_images must be in 1..65535");
    if (n < 0) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "n must be >= 0");
    if (n > 0 && !atoms) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "atoms must be non-NULL");
    const int kind = desc->kind;
    if (kind < IDIWF_EMIT_SPHERE || kind > IDIWF_EMIT_FIXED) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "unknown kind");
    if ((kind == IDIWF_EMIT_SITES || kind == IDIWF_EMIT_FIXED) && !desc->sites)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "sites must be non-NULL");
    if (kind == IDIWF_EMIT_FIXED && desc->n_sites != n)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "FIXED needs n_sites == n");
    if (kind == IDIWF_EMIT_SITES && desc->n_sites <= 0)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "SITES needs n_sites > 0");
    if (kind == IDIWF_EMIT_SITES && desc->n_sites > ((int64_t)1 << 40))
        return set_error(IDIWF_ERR_UNSUPPORTED, "at most 2^40 sites");
    if (kind == IDIWF_EMIT_SITES && desc->orientation == IDIWF_ORIENT_AXIS &&
        !(desc->axis[0] * desc->axis[0] + desc->axis[1] * desc->axis[1] + desc->axis[2] * desc->axis[2] > 0))
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "axis must be nonzero");
    if (kind == IDIWF_EMIT_GNORM || kind == IDIWF_EMIT_FOIL || (kind == IDIWF_EMIT_SITES && desc->weighted)) {
        const int na = kind == IDIWF_EMIT_FOIL ? 2 : 3;
        for (int a = 0; a < na; ++a)
            if (!(desc->fwhm[a] > 0) || !(desc->rho[a] > 0) || !std::isfinite(desc->fwhm[a]) ||
                !std::isfinite(desc->rho[a]))
                return set_error(IDIWF_ERR_INVALID_ARGUMENT, "fwhm and rho must be positive and finite");
    }
    if (!workspace || workspace_bytes < emitters_ws_bytes(desc, n_images))
        return set_error(IDIWF_ERR_WORKSPACE, "workspace smaller than idiwf_emitters_workspace_size()");
    if (reinterpret_cast<uintptr_t>(workspace) & 255)
        return set_error(IDIWF_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    WsHeader *hdr = static_cast<WsHeader *>(workspace);
    IDIWF_CUDA_CHECK(cudaMemsetAsync(workspace, 0, 2 * sizeof(uint32_t), stream));
    if (n == 0) return IDIWF_OK;

    EmitParams P{};
    P.kind = kind;
    P.random_phase = desc->random_phase;
    P.orientation = desc->orientation;
    P.weighted = desc->weighted;
    P.r = desc->r;
    for (int a = 0; a < 3; ++a) {
        P.fwhm[a] = desc->fwhm[a];
        P.rho[a] = desc->rho[a];
        P.s[a] = desc->weighted ? kLn2 * std::pow(2.0 / desc->fwhm[a], desc->rho[a]) : 0.0;
        P.axis[a] = desc->axis[a];
    }
    P.depth = desc->depth;
    P.attenuation = desc->attenuation;
    for (int i = 0; i < 9; ++i) P.rot[i] = desc->rot[i];
    P.sites = desc->sites;
    P.n_sites = desc->n_sites;
    P.n = n;
    P.k0 = rng->key[0];
    P.k1 = rng->key[1];
    P.stream = rng->stream;
    P.img0 = rng->first_image;

    const int sms = emit_sms();
    if (kind != IDIWF_EMIT_SITES) {
        const int gx = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)8 * sms / n_images + 1));
        const dim3 grid(gx, n_images);
        switch (kind) {
            case IDIWF_EMIT_SPHERE: emit_kernel<IDIWF_EMIT_SPHERE><<<grid, 256, 0, stream>>>(P, atoms, &hdr->error); break;
            case IDIWF_EMIT_GNORM: emit_kernel<IDIWF_EMIT_GNORM><<<grid, 256, 0, stream>>>(P, atoms, &hdr->error); break;
            case IDIWF_EMIT_FOIL: emit_kernel<IDIWF_EMIT_FOIL><<<grid, 256, 0, stream>>>(P, atoms, &hdr->error); break;
            default: emit_kernel<IDIWF_EMIT_FIXED><<<grid, 256, 0, stream>>>(P, atoms, &hdr->error); break;
        }
        IDIWF_CUDA_CHECK(cudaGetLastError());
        return IDIWF_OK;
    }
    double *rots = reinterpret_cast<double *>(static_cast<char *>(workspace) + 256);
    uint64_t *keys = reinterpret_cast<uint64_t *>(static_cast<char *>(workspace) + 256 +
                                                  align256((size_t)n_images * 9 * sizeof(double)));
    sites_rot_kernel<<<(n_images + 127) / 128, 128, 0, stream>>>(P, n_images, rots);
    IDIWF_CUDA_CHECK(cudaGetLastError());
    const int gx = (int)std::max<int64_t>(1, std::min<int64_t>((P.n_sites + 255) / 256, (int64_t)8 * sms / n_images + 1));
    for (int64_t base = 0, round = 0; base < n; base += P.n_sites, ++round) {
        const int64_t take = std::min<int64_t>(P.n_sites, n - base);
        sites_key_kernel<<<dim3(gx, n_images), 256, 0, stream>>>(P, (int)round, rots, keys);
        sites_select_kernel<<<n_images, kSelThreads, 0, stream>>>(P, take, base, rots, keys, atoms, &hdr->error);
        IDIWF_CUDA_CHECK(cudaGetLastError());
    }
    return IDIWF_OK;
}
