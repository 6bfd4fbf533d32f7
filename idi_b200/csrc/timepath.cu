// Time-dependent direct sum for sm_100a (FP64).
//
// Per pixel p (reference: idi/simulation/time.py:48-98, simtime.cu:50-148):
//   t_j   = -s_j / c + t0_j          s_j = (d/|d| - zhat) . r_j   (far field)
//   a_j   = exp(-i (s_j k - psi_j)) [ / |d| ]
//   sort (t_j, a_j) by t_j
//   x_0 = a_0,  x_m = a_m + exp(-(t_m - t_{m-1})/tau) x_{m-1}
//   I_p = sum_{m<n-1} -tau/2 |x_m|^2 expm1(-2 (t_{m+1}-t_m)/tau) + tau/2 |x_{n-1}|^2
//
// One CTA (512 threads) handles one pixel at a time (persistent, atomic
// pixel queue).  Arrival times are computed in FP64 with the exact rounding
// sequence of the reference (np.inner as fma(q2,z,fma(q1,y,q0*x)), IEEE
// division by c), so the keys -- and therefore the sorted order -- are bit
// for bit those of the reference.  The sort is an on-chip LSD radix sort
// (8 passes of 8 bits over the order-preserving 64-bit image of the double
// keys) that moves only 16-bit emitter indices: keys stay in a shared-memory
// table indexed by emitter, so N <= 20480 fits in 200 KB of shared memory.
// Ranking is per warp with __match_any_sync, which keeps the sort stable
// (ties, which the reference breaks arbitrarily, keep emitter order).  The
// decaying scan is a block-wide scan of affine maps x -> D x + B; the
// interval integral is a block reduction.

#include <algorithm>
#include <cmath>

#include "idiwf_internal.cuh"

namespace idiwf {

constexpr int kTimeThreads = 512;
constexpr int kTimeWarps = kTimeThreads / 32;
constexpr int kTimeIPT = 40;                                 // items per thread
constexpr int kTimeMaxN = kTimeThreads * kTimeIPT;           // 20480
constexpr size_t kTimeSmem = (size_t)kTimeMaxN * 8           // key table
                             + (size_t)kTimeMaxN * 2         // permutation
                             + (size_t)kTimeWarps * 256 * 4  // per-warp digit counters
                             + 256 * 4 + 1024;               // digit bases + scan scratch

__device__ __forceinline__ uint64_t sortable(double v) {
    const uint64_t b = (uint64_t)__double_as_longlong(v);
    return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

struct Affine {
    double d, br, bi;
};
// apply `first` then `second`
__device__ __forceinline__ Affine compose(const Affine &first, const Affine &second) {
    Affine r;
    r.d = second.d * first.d;
    r.br = fma(second.d, first.br, second.br);
    r.bi = fma(second.d, first.bi, second.bi);
    return r;
}

template <bool NF, bool SCALE>
__device__ __forceinline__ void arrival(const GeomParams &g, double dx, double dy, double dz, double dn,
                                        double q0, double q1, double q2, const double4 &a, double t0,
                                        double c, double &t, double &s_out, double &dist_out) {
    if (!NF) {
        const double s = __fma_rn(q2, a.z, __fma_rn(q1, a.y, __dmul_rn(q0, a.x)));
        t = __dadd_rn(__ddiv_rn(-s, c), t0);
        s_out = s;
        dist_out = dn;
    } else {
        const double ax = __dsub_rn(dx, a.x), ay = __dsub_rn(dy, a.y), az = __dsub_rn(dz, a.z);
        const double dist = __dsqrt_rn(__fma_rn(az, az, __fma_rn(ax, ax, __dmul_rn(ay, ay))));
        const double s = __dadd_rn(__dsub_rn(dist, dn), a.z);
        t = __dadd_rn(__ddiv_rn(s, c), t0);
        s_out = s;
        dist_out = dist;
    }
}

template <bool NF, bool SCALE>
__device__ __forceinline__ void amplitude(double k, double s, double psi, double dist, double &re, double &im) {
    double th;
    if (!NF) th = -__dsub_rn(__dmul_rn(s, k), psi);  // time.py:94 exp(-1j*(s*k-phases))
    else th = __dadd_rn(__dmul_rn(s, k), psi);       // simtime.cu:71 phase = s*k + w
    double sn, cs;
    sincos(th, &sn, &cs);
    if (SCALE) {
        cs = __ddiv_rn(cs, dist);
        sn = __ddiv_rn(sn, dist);
    }
    re = cs;
    im = sn;
}

template <bool NF, bool SCALE>
__global__ void __launch_bounds__(kTimeThreads, 1) time_kernel(const GeomParams g, const double *__restrict__ atoms,
                                                                const double *__restrict__ times, int n, double c,
                                                                double tau, double *__restrict__ out,
                                                                WsHeader *__restrict__ hdr, int order_pixel,
                                                                int *__restrict__ order_out,
                                                                double *__restrict__ keys_out) {
    extern __shared__ __align__(16) unsigned char smem[];
    double *keytab = reinterpret_cast<double *>(smem);
    uint16_t *perm = reinterpret_cast<uint16_t *>(smem + (size_t)kTimeMaxN * 8);
    uint32_t *H = reinterpret_cast<uint32_t *>(smem + (size_t)kTimeMaxN * 10);
    uint32_t *base = H + kTimeWarps * 256;
    double *scratch = reinterpret_cast<double *>(base + 256);  // 128 doubles
    __shared__ int s_pix;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int npix = g.nx * g.ny;
    const int S = 32 * kTimeIPT;  // elements per warp segment
    const uint32_t lt_mask = (1u << lane) - 1u;

    // order_pixel >= 0: process that one pixel only, record its sorted order
    // and write its intensity to out[0]
    int iter = 0;
    for (;;) {
        __syncthreads();
        if (tid == 0)
            s_pix = order_pixel >= 0 ? (iter == 0 ? order_pixel : npix) : (int)atomicAdd(&hdr->work_counter, 1u);
        __syncthreads();
        ++iter;
        const int p = s_pix;
        if (p >= npix) break;
        const int ix = p / g.ny, iy = p - ix * g.ny;
        double dx, dy, dz;
        pixel_time(g, ix, iy, dx, dy, dz);
        // time.py:89-91 (np.linalg.norm = sqrt((x*x + y*y) + z*z); q = det/d; q_z -= 1)
        const double dn = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
        const double q0 = __ddiv_rn(dx, dn), q1 = __ddiv_rn(dy, dn), q2 = __dsub_rn(__ddiv_rn(dz, dn), 1.0);

        // ---- keys: table by emitter index, +inf padding ----
        for (int j = tid; j < kTimeMaxN; j += kTimeThreads) {
            double t = __longlong_as_double(0x7FF0000000000000ll);  // +inf
            if (j < n) {
                const double4 a = reinterpret_cast<const double4 *>(atoms)[j];
                double s, dist;
                arrival<NF, SCALE>(g, dx, dy, dz, dn, q0, q1, q2, a, times[j], c, t, s, dist);
            }
            keytab[j] = t;
        }
        // initial order: warp segment layout, element (i, lane) of warp w at
        // position w*S + i*32 + lane holds emitter w*S + i*32 + lane
        uint16_t idx[kTimeIPT];
#pragma unroll
        for (int i = 0; i < kTimeIPT; ++i) idx[i] = (uint16_t)(warp * S + i * 32 + lane);
        __syncthreads();

        for (int pass = 0; pass < 8; ++pass) {
            const int shift = pass * 8;
            uint32_t *Hw = H + warp * 256;
            for (int k = lane; k < 256; k += 32) Hw[k] = 0;
            __syncwarp();
            // phase 1: per-warp digit histogram
#pragma unroll 4
            for (int i = 0; i < kTimeIPT; ++i) {
                const uint32_t dg = (uint32_t)(sortable(keytab[idx[i]]) >> shift) & 255u;
                const uint32_t peers = __match_any_sync(0xffffffffu, dg);
                if ((peers & lt_mask) == 0) Hw[dg] += __popc(peers);
                __syncwarp();
            }
            __syncthreads();
            // digit totals and exclusive prefix over warps, then over digits
            if (tid < 256) {
                uint32_t run = 0;
                for (int w = 0; w < kTimeWarps; ++w) {
                    const uint32_t h = H[w * 256 + tid];
                    H[w * 256 + tid] = run;
                    run += h;
                }
                base[tid] = run;
            }
            __syncthreads();
            if (warp == 0) {
                // exclusive scan of 256 digit totals, 8 per lane
                uint32_t v[8], sum = 0;
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    v[k] = base[lane * 8 + k];
                    sum += v[k];
                }
                uint32_t incl = sum;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += y;
                }
                uint32_t run = incl - sum;
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    base[lane * 8 + k] = run;
                    run += v[k];
                }
            }
            __syncthreads();
            for (int k = lane; k < 256; k += 32) Hw[k] += base[k];
            __syncwarp();
            // phase 2: stable scatter of indices
#pragma unroll 4
            for (int i = 0; i < kTimeIPT; ++i) {
                const uint32_t dg = (uint32_t)(sortable(keytab[idx[i]]) >> shift) & 255u;
                const uint32_t peers = __match_any_sync(0xffffffffu, dg);
                const uint32_t b0 = Hw[dg];
                const uint32_t rank = b0 + __popc(peers & lt_mask);
                __syncwarp();
                if ((peers & lt_mask) == 0) Hw[dg] = b0 + __popc(peers);
                __syncwarp();
                perm[rank] = idx[i];
            }
            __syncthreads();
#pragma unroll
            for (int i = 0; i < kTimeIPT; ++i) idx[i] = perm[warp * S + i * 32 + lane];
            __syncthreads();
        }
        // perm[m] = emitter at sorted position m (positions >= n hold padding)

        if (p == order_pixel) {
            for (int m = tid; m < n; m += kTimeThreads) {
                order_out[m] = perm[m];
                keys_out[m] = keytab[perm[m]];
            }
        }

        // ---- decaying scan over the sorted sequence (blocked: thread owns
        //      positions [tid*IPT, tid*IPT + IPT)) ----
        const int m0 = tid * kTimeIPT;
        Affine agg = {1.0, 0.0, 0.0};
        for (int i = 0; i < kTimeIPT; ++i) {
            const int m = m0 + i;
            if (m >= n) break;
            const int j = perm[m];
            const double4 a = reinterpret_cast<const double4 *>(atoms)[j];
            double t, s, dist, re, im;
            arrival<NF, SCALE>(g, dx, dy, dz, dn, q0, q1, q2, a, times[j], c, t, s, dist);
            amplitude<NF, SCALE>(g.k, s, a.w, dist, re, im);
            const double dec = m == 0 ? 0.0 : exp(__ddiv_rn(-__dsub_rn(keytab[j], keytab[perm[m - 1]]), tau));
            const Affine e = {dec, re, im};
            agg = compose(agg, e);
        }
        // block exclusive scan of aggregates
        Affine incl = agg;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            Affine y;
            y.d = __shfl_up_sync(0xffffffffu, incl.d, o);
            y.br = __shfl_up_sync(0xffffffffu, incl.br, o);
            y.bi = __shfl_up_sync(0xffffffffu, incl.bi, o);
            if (lane >= o) incl = compose(y, incl);
        }
        if (lane == 31) {
            scratch[warp * 3 + 0] = incl.d;
            scratch[warp * 3 + 1] = incl.br;
            scratch[warp * 3 + 2] = incl.bi;
        }
        __syncthreads();
        Affine wpre = {1.0, 0.0, 0.0};  // composition of all earlier warps
        for (int w = 0; w < warp; ++w) {
            const Affine y = {scratch[w * 3 + 0], scratch[w * 3 + 1], scratch[w * 3 + 2]};
            wpre = compose(wpre, y);
        }
        Affine excl;
        excl.d = __shfl_up_sync(0xffffffffu, incl.d, 1);
        excl.br = __shfl_up_sync(0xffffffffu, incl.br, 1);
        excl.bi = __shfl_up_sync(0xffffffffu, incl.bi, 1);
        if (lane == 0) excl = Affine{1.0, 0.0, 0.0};
        excl = compose(wpre, excl);
        // x entering this thread's run = excl applied to x_{-1} = 0
        double xr = excl.br, xi = excl.bi;
        double part = 0.0;
        for (int i = 0; i < kTimeIPT; ++i) {
            const int m = m0 + i;
            if (m >= n) break;
            const int j = perm[m];
            const double4 a = reinterpret_cast<const double4 *>(atoms)[j];
            double t, s, dist, re, im;
            arrival<NF, SCALE>(g, dx, dy, dz, dn, q0, q1, q2, a, times[j], c, t, s, dist);
            amplitude<NF, SCALE>(g.k, s, a.w, dist, re, im);
            if (m == 0) {
                xr = re;
                xi = im;
            } else {
                const double dec = exp(__ddiv_rn(-__dsub_rn(keytab[j], keytab[perm[m - 1]]), tau));
                xr = __dadd_rn(re, __dmul_rn(dec, xr));
                xi = __dadd_rn(im, __dmul_rn(dec, xi));
            }
            const double I = __dadd_rn(__dmul_rn(xi, xi), __dmul_rn(xr, xr));
            if (m < n - 1) {
                const double td = __dsub_rn(keytab[perm[m + 1]], keytab[j]);
                part += __dmul_rn(__dmul_rn(-tau / 2, I), expm1(__ddiv_rn(-2 * td, tau)));
            } else {
                part += tau / 2 * I;
            }
        }
        // block sum
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
        __syncthreads();
        if (lane == 0) scratch[64 + warp] = part;
        __syncthreads();
        if (tid == 0) {
            double tot = 0.0;
            for (int w = 0; w < kTimeWarps; ++w) tot += scratch[64 + w];
            out[order_pixel >= 0 ? 0 : p] = tot;
        }
    }
}

template <bool NF, bool SCALE>
static void *time_kernel_ptr() {
    return (void *)time_kernel<NF, SCALE>;
}

static idiwf_status time_validate(const idiwf_geom *geom, const double *atoms, const double *times, int64_t n,
                                  double c, double tau) {
    if (!geom || geom->nx <= 0 || geom->ny <= 0 || (int64_t)geom->nx * geom->ny >= ((int64_t)1 << 31))
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "bad detector size");
    if (geom->offset[0] != 0.0 || geom->offset[1] != 0.0)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "the time path has no detector offset");
    if (geom->flags & IDIWF_SECONDORDER)
        return set_error(IDIWF_ERR_UNSUPPORTED, "secondorder is not defined for the time path");
    if (n < 1) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "the time path needs at least one emitter");
    if (n > kTimeMaxN) return set_error(IDIWF_ERR_UNSUPPORTED, "too many emitters for the on-chip sort");
    if (!atoms || !times) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "atoms/times are NULL");
    if (reinterpret_cast<uintptr_t>(atoms) & 31) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "atoms must be 32-byte aligned");
    if (!(c > 0) || !(tau > 0)) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "c and tau must be positive");
    return IDIWF_OK;
}

static idiwf_status time_launch(const idiwf_geom *geom, const double *atoms, const double *times, int64_t n,
                                double c, double tau, double *out, void *workspace, size_t workspace_bytes,
                                int order_pixel, int *order_out, double *keys_out, cudaStream_t stream) {
    if (!workspace || workspace_bytes < kWsDataOffset)
        return set_error(IDIWF_ERR_WORKSPACE, "workspace smaller than idiwf_time_workspace_size()");
    if (reinterpret_cast<uintptr_t>(workspace) & 255)
        return set_error(IDIWF_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    WsHeader *hdr = static_cast<WsHeader *>(workspace);
    const GeomParams g = make_geom(geom);
    const bool nf = geom->flags & IDIWF_NF, sc = geom->flags & IDIWF_SCALE;
    void *fn = nf ? (sc ? time_kernel_ptr<true, true>() : time_kernel_ptr<true, false>())
                  : (sc ? time_kernel_ptr<false, true>() : time_kernel_ptr<false, false>());
    IDIWF_CUDA_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTimeSmem));
    IDIWF_CUDA_CHECK(cudaMemsetAsync(hdr, 0, 2 * sizeof(uint32_t), stream));  // counter + error word
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int npix = geom->nx * geom->ny;
    const int grid = order_pixel >= 0 ? 1 : std::min(npix, sms);
    int ni = (int)n;
    void *args[] = {(void *)&g, &atoms, &times, &ni, &c, &tau, &out, &hdr, &order_pixel, &order_out, &keys_out};
    IDIWF_CUDA_CHECK(cudaLaunchKernel(fn, dim3(grid), dim3(kTimeThreads), args, kTimeSmem, stream));
    return IDIWF_OK;
}

}  // namespace idiwf

using namespace idiwf;

extern "C" int64_t idiwf_time_max_emitters(void) { return kTimeMaxN; }

extern "C" size_t idiwf_time_workspace_size(const idiwf_geom *geom, int64_t n) {
    (void)geom;
    (void)n;
    return kWsDataOffset;
}

extern "C" idiwf_status idiwf_time_forward(const idiwf_geom *geom, const double *atoms, const double *times,
                                           int64_t n, double c, double tau, double *out, void *workspace,
                                           size_t workspace_bytes, cudaStream_t stream) {
    idiwf_status st = time_validate(geom, atoms, times, n, c, tau);
    if (st != IDIWF_OK) return st;
    if (!out) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "out is NULL");
    return time_launch(geom, atoms, times, n, c, tau, out, workspace, workspace_bytes, -1, nullptr, nullptr, stream);
}

extern "C" idiwf_status idiwf_time_order(const idiwf_geom *geom, const double *atoms, const double *times,
                                         int64_t n, double c, int32_t ix, int32_t iy, int32_t *order,
                                         double *sorted_keys, void *workspace, size_t workspace_bytes,
                                         cudaStream_t stream) {
    idiwf_status st = time_validate(geom, atoms, times, n, c, 1.0);
    if (st != IDIWF_OK) return st;
    if (!order || !sorted_keys) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "order/sorted_keys are NULL");
    if (ix < 0 || iy < 0 || ix >= geom->nx || iy >= geom->ny)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "pixel outside the detector");
    if (!workspace || workspace_bytes < kWsDataOffset)
        return set_error(IDIWF_ERR_WORKSPACE, "workspace smaller than idiwf_time_workspace_size()");
    // the intensity of the pixel goes to a scratch slot of the workspace header
    double *scratch = reinterpret_cast<double *>(&static_cast<WsHeader *>(workspace)->pad[0]);
    return time_launch(geom, atoms, times, n, c, 1.0, scratch, workspace, workspace_bytes, ix * geom->ny + iy, order,
                       sorted_keys, stream);
}
