// Elementwise steps of the FFT autocorrelation (idi/reconstruction/cusimple.py):
// the power spectrum in place, the fftshift + centre crop fused with the
// normalisation, and the correlator's running mean / variance.  HBM-bound,
// one pass each; the transforms themselves are cuFFT's.
#include <cmath>

#include "idiwf_internal.cuh"

namespace idiwf {

template <typename T>
__global__ void power_kernel(T *__restrict__ z, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const T re = z[2 * i], im = z[2 * i + 1];
        z[2 * i] = re * re + im * im;
        z[2 * i + 1] = T(0);
    }
}

struct CropDims {
    int32_t ndim;
    int32_t g[3], n[3];  // full and half-output extents, trailing axes
};

template <typename T>
__global__ void crop_kernel(const T *__restrict__ full, int64_t batch, const CropDims D, const T *__restrict__ norm,
                            int mode, T threshold, T *__restrict__ out) {
    int64_t per_out = 1, per_full = 1;
    for (int k = 0; k < D.ndim; ++k) {
        per_out *= 2 * D.n[k];
        per_full *= D.g[k];
    }
    const int64_t total = per_out * batch;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = t / per_out;
        int64_t r = t - b * per_out;
        int64_t src = 0;
        int64_t stride = 1;
        for (int k = D.ndim - 1; k >= 0; --k) {
            const int e = 2 * D.n[k];
            const int i = (int)(r % e);
            r /= e;
            int j = (i - D.n[k]) % D.g[k];
            if (j < 0) j += D.g[k];
            src += (int64_t)j * stride;
            stride *= D.g[k];
        }
        T y = full[b * per_full + src];
        if (norm) {
            const T c = norm[t - b * per_out];
            if (mode == 0)
                y = c < threshold ? T(NAN) : y / c;
            else
                y = c > threshold ? y / c : T(0);
        }
        out[t] = y;
    }
}

__global__ void welford_kernel(const float *__restrict__ x, float *__restrict__ mean, float *__restrict__ nvar,
                               int64_t n, int64_t count) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float v = x[i];
        if (count == 1) {
            mean[i] = v;
            nvar[i] = 0.0f;
        } else {
            const float delta = v - mean[i];
            const float m = mean[i] + delta / (float)count;
            mean[i] = m;
            nvar[i] = nvar[i] + delta * (v - m);
        }
    }
}

static int ew_blocks(int64_t n) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sms * 16));
}

}  // namespace idiwf

using namespace idiwf;

extern "C" idiwf_status idiwf_power_spectrum(void *spectrum, int64_t n, int32_t dtype, cudaStream_t stream) {
    if (n < 0 || (n > 0 && !spectrum)) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "bad spectrum");
    if (n == 0) return IDIWF_OK;
    if (dtype == IDIWF_F64)
        power_kernel<double><<<ew_blocks(n), 256, 0, stream>>>(static_cast<double *>(spectrum), n);
    else if (dtype == IDIWF_F32)
        power_kernel<float><<<ew_blocks(n), 256, 0, stream>>>(static_cast<float *>(spectrum), n);
    else
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "dtype must be IDIWF_F64 or IDIWF_F32");
    IDIWF_CUDA_CHECK(cudaGetLastError());
    return IDIWF_OK;
}

extern "C" idiwf_status idiwf_corr_crop(const void *full, int32_t dtype, int64_t batch, int32_t ndim, const int32_t *g,
                                        const int32_t *n, const void *norm, int32_t mode, double threshold, void *out,
                                        cudaStream_t stream) {
    if (!full || !out || !g || !n) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "NULL argument");
    if (ndim < 1 || ndim > 3) return set_error(IDIWF_ERR_UNSUPPORTED, "1 to 3 correlated axes");
    if (batch <= 0) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "batch must be positive");
    if (mode != 0 && mode != 1) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "mode must be 0 or 1");
    CropDims D{};
    D.ndim = ndim;
    int64_t total = batch;
    for (int k = 0; k < ndim; ++k) {
        if (g[k] <= 0 || n[k] <= 0) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "extents must be positive");
        D.g[k] = g[k];
        D.n[k] = n[k];
        total *= 2 * (int64_t)n[k];
    }
    if (dtype == IDIWF_F64)
        crop_kernel<double><<<ew_blocks(total), 256, 0, stream>>>(static_cast<const double *>(full), batch, D,
                                                                  static_cast<const double *>(norm), mode, threshold,
                                                                  static_cast<double *>(out));
    else if (dtype == IDIWF_F32)
        crop_kernel<float><<<ew_blocks(total), 256, 0, stream>>>(static_cast<const float *>(full), batch, D,
                                                                 static_cast<const float *>(norm), mode,
                                                                 (float)threshold, static_cast<float *>(out));
    else
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "dtype must be IDIWF_F64 or IDIWF_F32");
    IDIWF_CUDA_CHECK(cudaGetLastError());
    return IDIWF_OK;
}

extern "C" idiwf_status idiwf_welford_update(const float *x, float *mean, float *nvar, int64_t n, int64_t count,
                                             cudaStream_t stream) {
    if (n < 0 || count < 1 || (n > 0 && (!x || !mean || !nvar)))
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "bad arguments");
    if (n == 0) return IDIWF_OK;
    welford_kernel<<<ew_blocks(n), 256, 0, stream>>>(x, mean, nvar, n, count);
    IDIWF_CUDA_CHECK(cudaGetLastError());
    return IDIWF_OK;
}
