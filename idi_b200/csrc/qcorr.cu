// Direct q-space autocorrelation of detector images (the consumers of the
// simulated intensities): idi/reconstruction/cucorrad.py (radial) and
// idi/reconstruction/cucor.py (3d).
//
// Pair set (both): reference pixel (r, c), target (r + dr, c + dc) with
// 0 <= dr < qmax and dc in the column-offset range; one thread per column
// offset walks the row pair and keeps a run: consecutive pairs with the same
// bin are summed in FP32 and the run is added to the FP64 histogram when the
// bin changes -- the radial reference kernel's accumulation, and for the 3d
// one (which adds every pair to FP32 bins) far fewer atomics.
//
//  * qcorr_radial_kernel — CTA = (reference row, group of kRowsPerCta target
//    rows, image).  The reference row and each target row are staged in
//    shared memory as float4 {qx, qy, qz, v}: one broadcast LDS.128 and one
//    conflict-free LDS.128 per pair.  The bin round(sqrt(d2)) is re-derived
//    only when d2 leaves the current bin's interval (a table of the exact
//    d2 thresholds), since it rarely changes along a row.  Bins go to an FP64
//    shared-memory histogram, added to the output once per CTA.
//  * qcorr_3d_kernel — the same walk over float2 {zd, v} rows; runs go to the
//    FP64 output with global atomics (the 3d histogram does not fit on chip);
//    bins outside the array are dropped.
//  * qcorr_sym_kernel — the reference's symmetrisation about the centre, each
//    mirror pair handled by exactly one thread.
#include <cmath>

#include "idiwf_internal.cuh"

namespace idiwf {

constexpr int kRowsPerCta = 8;
constexpr int kQcorrMaxSmemCols = 4096;

// ---------------------------------------------------------------------------
// radial
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) qcorr_radial_kernel(const float4 *__restrict__ q,
                                                            const float *__restrict__ images, int nr, int nc,
                                                            int qmax, double *__restrict__ out) {
    extern __shared__ __align__(16) unsigned char qsm[];
    float4 *sref = reinterpret_cast<float4 *>(qsm);
    float4 *stgt = sref + nc;
    double *hist = reinterpret_cast<double *>(stgt + nc);
    float *bound = reinterpret_cast<float *>(hist + qmax + 1);  // qmax + 3 entries
    const int refr = blockIdx.x;
    const int img = blockIdx.z;
    const float *v = images + (int64_t)img * nr * nc;
    const int tid = threadIdx.x;
    for (int i = tid; i <= qmax; i += blockDim.x) hist[i] = 0.0;
    // bound[k]: smallest float d2 >= 0 with rint(sqrt(d2)) >= k, k = 0..qmax+1,
    // by bisection over the (monotone) float bit patterns with the very
    // operations of the bin below; bound[qmax+2] = +inf.  Bins above qmax are
    // one class (the reference only tests dq <= qmax and dq < qmax there).
    for (int k = tid; k <= qmax + 2; k += blockDim.x) {
        float b;
        if (k == 0) {
            b = 0.0f;
        } else if (k == qmax + 2) {
            b = __int_as_float(0x7F800000);
        } else {
            uint32_t lo = 0u, hi = 0x7F800000u;  // rint(sqrt(+0)) = 0 < k <= rint(sqrt(+inf))
            while (hi - lo > 1u) {
                const uint32_t mid = lo + (hi - lo) / 2u;
                if ((int)rintf(__fsqrt_rn(__uint_as_float(mid))) >= k) hi = mid;
                else lo = mid;
            }
            b = __uint_as_float(hi);
        }
        bound[k] = b;
    }
    for (int c = tid; c < nc; c += blockDim.x) {
        float4 a = q[(int64_t)refr * nc + c];
        a.w = v[(int64_t)refr * nc + c];
        sref[c] = a;
    }
    const int offsetc = tid - qmax;
    const bool active = tid < 2 * qmax + 1;
    const int c0 = max(0, -offsetc), c1 = min(nc, nc - offsetc);  // tc = refc + offsetc in [0, nc)
    const int dr0 = blockIdx.y * kRowsPerCta;
    for (int dr = dr0; dr < min(dr0 + kRowsPerCta, qmax); ++dr) {
        const int tr = refr + dr;
        if (tr >= nr) break;
        __syncthreads();
        for (int c = tid; c < nc; c += blockDim.x) {
            float4 b = q[(int64_t)tr * nc + c];
            b.w = v[(int64_t)tr * nc + c];
            stgt[c] = b;
        }
        __syncthreads();
        if (active) {
            float val = 0.0f;
            int dqold = tid / 2;  // the reference's initial run bin (receives an empty run)
            int dq = qmax + 1;
            float lo = 1.0f, hi = 0.0f;  // empty: the first pair derives its bin
            // The reference, per pair: if dq <= qmax { if dq != dqold { add the
            // run to dqold; dqold = dq; val = 0 } val += v v' }.  While the bin
            // stays the same, dq == dqold whenever dq <= qmax, so that test
            // only needs to run when the bin changes.
            bool in_range = false;
#pragma unroll 4
            for (int refc = c0; refc < c1; ++refc) {
                const float4 a = sref[refc];
                const float4 b = stgt[refc + offsetc];
                const float dx = __fsub_rn(a.x, b.x), dy = __fsub_rn(a.y, b.y), dz = __fsub_rn(a.z, b.z);
                const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
                if (!(d2 >= lo && d2 < hi)) {  // left the current bin's interval
                    dq = min((int)rintf(__fsqrt_rn(d2)), qmax + 1);
                    lo = bound[dq];
                    hi = bound[dq + 1];
                    in_range = dq <= qmax;
                    if (in_range && dq != dqold) {
                        atomicAdd(&hist[dqold], (double)val);
                        dqold = dq;
                        val = 0.0f;
                    }
                }
                if (in_range) val = __fadd_rn(val, __fmul_rn(a.w, b.w));
            }
            if (dq < qmax) atomicAdd(&hist[dq], (double)val);
        }
    }
    __syncthreads();
    double *o = out + (int64_t)img * qmax;
    for (int i = tid; i < qmax; i += blockDim.x)
        if (hist[i] != 0.0) atomicAdd(&o[i], hist[i]);
}

// ---------------------------------------------------------------------------
// 3d
// ---------------------------------------------------------------------------
struct Q3Params {
    int nr, nc, qmax, maxdqz;
    float xcenter, ycenter, z;
};

__device__ __forceinline__ void q3_flush(double *o, int64_t bin, float val) {
    if (bin >= 0) atomicAdd(&o[bin], (double)val);
}

__global__ void __launch_bounds__(1024) qcorr_3d_kernel(const float *__restrict__ zd, const float *__restrict__ images,
                                                        const Q3Params P, double *__restrict__ out) {
    extern __shared__ __align__(16) unsigned char qsm[];
    float2 *sref = reinterpret_cast<float2 *>(qsm);
    float2 *stgt = sref + P.nc;
    const int refr = blockIdx.x;
    const int img = blockIdx.z;
    const int nc = P.nc, qmax = P.qmax;
    const int D0 = 2 * P.maxdqz, D1 = 2 * qmax, D2 = 2 * qmax;
    const float *v = images + (int64_t)img * P.nr * nc;
    double *o = out + (int64_t)img * D0 * D1 * D2;
    const int tid = threadIdx.x;
    for (int c = tid; c < nc; c += blockDim.x)
        sref[c] = make_float2(zd[(int64_t)refr * nc + c], v[(int64_t)refr * nc + c]);
    const float refr2 = __fsub_rn((float)refr, P.xcenter);
    const int dr0 = blockIdx.y * kRowsPerCta;
    for (int dr = dr0; dr < min(dr0 + kRowsPerCta, qmax); ++dr) {
        const int tr = refr + dr;
        if (tr >= P.nr) break;
        __syncthreads();
        for (int c = tid; c < nc; c += blockDim.x)
            stgt[c] = make_float2(zd[(int64_t)tr * nc + c], v[(int64_t)tr * nc + c]);
        __syncthreads();
        const float tr2 = __fsub_rn((float)tr, P.xcenter);
        for (int offsetc = tid - (qmax - 1); offsetc <= qmax - 1; offsetc += blockDim.x) {
            const int c0 = max(0, -offsetc), c1 = min(nc, nc - offsetc);
            int64_t bin = -1;
            float val = 0.0f;
            for (int refc = c0; refc < c1; ++refc) {
                const int tc = refc + offsetc;
                const float2 a = sref[refc];
                const float2 b = stgt[tc];
                const int dqx = qmax + (int)rintf(__fsub_rn(__fmul_rn(tr2, b.x), __fmul_rn(refr2, a.x)));
                const int dqy = qmax + (int)rintf(__fsub_rn(__fmul_rn(__fsub_rn((float)tc, P.ycenter), b.x),
                                                            __fmul_rn(__fsub_rn((float)refc, P.ycenter), a.x)));
                const int dqz = P.maxdqz + (int)rintf(__fmul_rn(P.z, __fsub_rn(a.x, b.x)));
                if (dqz < 0 || dqz >= D0 || dqy < 0 || dqy >= D1 || dqx < 0 || dqx >= D2) continue;
                const int64_t nb = ((int64_t)dqz * D1 + dqy) * D2 + dqx;
                if (nb != bin) {
                    q3_flush(o, bin, val);
                    bin = nb;
                    val = 0.0f;
                }
                val = __fadd_rn(val, __fmul_rn(a.y, b.y));
            }
            q3_flush(o, bin, val);
        }
    }
}

// bins i and -i mod (D0, D1, D2) for i_x in [0, n2) hold the sum of both;
// one thread per mirror pair (the smaller index where both ends are
// visited), a bin that is its own mirror doubles.  n2 is the x extent the
// reference's assemble launch covers: D2/2, or 2 (D2/4) when D2 > 64.
__global__ void qcorr_sym_kernel(double *__restrict__ out, int D0, int D1, int D2, int n2, int n_images) {
    const int64_t per = (int64_t)D0 * D1 * n2;
    const int64_t total = per * n_images;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int img = (int)(t / per);
        int64_t r = t - (int64_t)img * per;
        const int i2 = (int)(r % n2);
        r /= n2;
        const int i1 = (int)(r % D1);
        const int i0 = (int)(r / D1);
        const int m0 = (D0 - i0) % D0, m1 = (D1 - i1) % D1, m2 = (D2 - i2) % D2;
        double *o = out + (int64_t)img * D0 * D1 * D2;
        const int64_t a = ((int64_t)i0 * D1 + i1) * D2 + i2;
        const int64_t b = ((int64_t)m0 * D1 + m1) * D2 + m2;
        if (a == b) {
            o[a] = 2.0 * o[a];
        } else if (m2 >= n2 || a < b) {  // the mirror is visited too only when m2 < n2: take one of the two
            const double s = o[a] + o[b];
            o[a] = s;
            o[b] = s;
        }
    }
}

static int qcorr_sms() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

}  // namespace idiwf

using namespace idiwf;

extern "C" size_t idiwf_qcorr_workspace_size(int32_t nr, int32_t nc) {
    (void)nr;
    (void)nc;
    return 256;
}

extern "C" idiwf_status idiwf_qcorr_radial(const float *q, const float *images, int32_t n_images, int32_t nr,
                                           int32_t nc, int32_t qmax, double *out, void *workspace,
                                           size_t workspace_bytes, cudaStream_t stream) {
    if (!q || !images || !out) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "q, images and out must be non-NULL");
    if (n_images <= 0 || n_images > 65535 || nr <= 0 || nc <= 0)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "n_images in 1..65535, nr and nc positive");
    if (qmax < 1 || qmax > 511) return set_error(IDIWF_ERR_UNSUPPORTED, "qmax must be in 1..511");
    if (nc > kQcorrMaxSmemCols) return set_error(IDIWF_ERR_UNSUPPORTED, "at most 4096 detector columns");
    if (reinterpret_cast<uintptr_t>(q) & 15) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "q must be 16-byte aligned");
    if (!workspace || workspace_bytes < 256) return set_error(IDIWF_ERR_WORKSPACE, "workspace too small");
    IDIWF_CUDA_CHECK(cudaMemsetAsync(out, 0, sizeof(double) * (size_t)n_images * qmax, stream));
    const int threads = ((2 * qmax + 1) + 31) / 32 * 32;
    const size_t smem = 2 * (size_t)nc * sizeof(float4) + (size_t)(qmax + 1) * sizeof(double) +
                        (size_t)(qmax + 3) * sizeof(float);
    IDIWF_CUDA_CHECK(cudaFuncSetAttribute(qcorr_radial_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const dim3 grid(nr, (qmax + kRowsPerCta - 1) / kRowsPerCta, n_images);
    qcorr_radial_kernel<<<grid, threads, smem, stream>>>(reinterpret_cast<const float4 *>(q), images, nr, nc, qmax,
                                                         out);
    IDIWF_CUDA_CHECK(cudaGetLastError());
    return IDIWF_OK;
}

extern "C" idiwf_status idiwf_qcorr_3d(const float *zd, const float *images, int32_t n_images, int32_t nr, int32_t nc,
                                       int32_t qmax, int32_t maxdqz, float xcenter, float ycenter, float z, double *out,
                                       void *workspace, size_t workspace_bytes, cudaStream_t stream) {
    if (!zd || !images || !out) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "zd, images and out must be non-NULL");
    if (n_images <= 0 || n_images > 65535 || nr <= 0 || nc <= 0)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "n_images in 1..65535, nr and nc positive");
    if (qmax < 1 || qmax > 1024) return set_error(IDIWF_ERR_UNSUPPORTED, "qmax must be in 1..1024");
    if (maxdqz < 1 || maxdqz > 4096) return set_error(IDIWF_ERR_UNSUPPORTED, "maxdqz must be in 1..4096");
    if (nc > 2 * kQcorrMaxSmemCols) return set_error(IDIWF_ERR_UNSUPPORTED, "at most 8192 detector columns");
    if (!workspace || workspace_bytes < 256) return set_error(IDIWF_ERR_WORKSPACE, "workspace too small");
    const int64_t D0 = 2 * (int64_t)maxdqz, D1 = 2 * (int64_t)qmax, D2 = 2 * (int64_t)qmax;
    IDIWF_CUDA_CHECK(cudaMemsetAsync(out, 0, sizeof(double) * (size_t)(n_images * D0 * D1 * D2), stream));
    Q3Params P{nr, nc, qmax, maxdqz, xcenter, ycenter, z};
    const size_t smem = 2 * (size_t)nc * sizeof(float2);
    IDIWF_CUDA_CHECK(cudaFuncSetAttribute(qcorr_3d_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int threads = std::min(1024, ((2 * qmax - 1) + 31) / 32 * 32);
    const dim3 grid(nr, (qmax + kRowsPerCta - 1) / kRowsPerCta, n_images);
    qcorr_3d_kernel<<<grid, threads, smem, stream>>>(zd, images, P, out);
    IDIWF_CUDA_CHECK(cudaGetLastError());
    const int n2 = (int)(D2 > 64 ? 2 * (D2 / 4) : D2 / 2);
    const int64_t pairs = n_images * D0 * D1 * n2;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((pairs + 255) / 256, 16 * (int64_t)qcorr_sms()));
    qcorr_sym_kernel<<<blocks, 256, 0, stream>>>(out, (int)D0, (int)D1, (int)D2, n2, n_images);
    IDIWF_CUDA_CHECK(cudaGetLastError());
    return IDIWF_OK;
}
