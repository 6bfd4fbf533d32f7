// Error reporting, diagnostics and the pipe-throughput microbenchmark.
#include <cstdio>
#include <string>

#include "idiwf_internal.cuh"

namespace idiwf {

static thread_local std::string g_last_error = "no error";

idiwf_status set_error(idiwf_status st, const std::string &msg) {
    g_last_error = msg;
    return st;
}

idiwf_status cuda_error(cudaError_t e, const char *where) {
    g_last_error = std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return IDIWF_ERR_CUDA;
}

// ---------------------------------------------------------------------------
// microbenchmarks: each thread runs independent dependency chains so the
// pipe, not latency, is the limit.  Results are folded into `sink` so the
// compiler cannot drop the work.
// ---------------------------------------------------------------------------
constexpr int kMbIters = 4096;

__global__ void mb_mufu(float *sink, float seed) {
    float a0 = seed + threadIdx.x * 1e-3f, a1 = a0 + 0.1f, a2 = a0 + 0.2f, a3 = a0 + 0.3f;
    float acc = 0.f;
#pragma unroll 4
    for (int i = 0; i < kMbIters; ++i) {
        float s0, c0, s1, c1, s2, c2, s3, c3;
        __sincosf(a0, &s0, &c0);
        __sincosf(a1, &s1, &c1);
        __sincosf(a2, &s2, &c2);
        __sincosf(a3, &s3, &c3);
        a0 = s0 + c1;
        a1 = s1 + c2;
        a2 = s2 + c3;
        a3 = s3 + c0;
    }
    acc = a0 + a1 + a2 + a3;
    if (acc == 12345.f) sink[threadIdx.x] = acc;
}

__global__ void mb_dfma(double *sink, double seed) {
    double a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = seed + k + threadIdx.x;
    const double m = 0.999999, c = 1e-7;
#pragma unroll 4
    for (int i = 0; i < kMbIters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = __fma_rn(a[k], m, c);
    }
    double s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == 12345.0) sink[threadIdx.x] = s;
}

__global__ void mb_ffma(float *sink, float seed) {
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = seed + k + threadIdx.x;
    const float m = 0.999999f, c = 1e-7f;
#pragma unroll 4
    for (int i = 0; i < kMbIters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = __fmaf_rn(a[k], m, c);
    }
    float s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == 12345.f) sink[threadIdx.x] = s;
}

__global__ void mb_ffma2(float *sink, float seed) {
    float2 a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = make_float2(seed + k + threadIdx.x, seed - k);
    const float2 m = make_float2(0.999999f, 0.999998f), c = make_float2(1e-7f, 2e-7f);
#pragma unroll 4
    for (int i = 0; i < kMbIters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = __ffma2_rn(a[k], m, c);
    }
    float s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k].x + a[k].y;
    if (s == 12345.f) sink[threadIdx.x] = s;
}

}  // namespace idiwf

using namespace idiwf;

extern "C" const char *idiwf_last_error_string(void) { return g_last_error.c_str(); }

extern "C" int32_t idiwf_version(void) { return (1 << 16) | 1; }

extern "C" idiwf_status idiwf_workspace_error(const void *workspace, cudaStream_t stream) {
    if (!workspace) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "workspace is NULL");
    WsHeader h;
    IDIWF_CUDA_CHECK(cudaMemcpyAsync(&h, workspace, sizeof(h), cudaMemcpyDeviceToHost, stream));
    IDIWF_CUDA_CHECK(cudaStreamSynchronize(stream));
    if (h.error & kErrTimeout) return set_error(IDIWF_ERR_TIMEOUT, "a bounded device wait gave up");
    if (h.error & kErrValue)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT,
                         "invalid input value (negative or NaN entry, all-zero image, or photon count mismatch)");
    if (h.error & kErrRange)
        return set_error(IDIWF_ERR_UNSUPPORTED,
                         "emitter coordinates too large for the split-precision phase range");
    if (h.error & kErrGeometry)
        return set_error(IDIWF_ERR_UNSUPPORTED,
                         "near-field geometry outside the split-precision range (emitters farther than a quarter "
                         "of the detector distance from the origin, or a path-difference remainder above 2 rad); "
                         "use the FP64 kernel (settings 'double' or 'accurate')");
    return IDIWF_OK;
}

extern "C" idiwf_status idiwf_microbench(int32_t kind, void *scratch, cudaStream_t stream, double *rate) {
    if (!scratch || !rate || kind < 0 || kind > 3) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "bad arguments");
    int dev = 0, sms = 0;
    IDIWF_CUDA_CHECK(cudaGetDevice(&dev));
    IDIWF_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int threads = 512, blocks = sms * 4;
    cudaEvent_t e0, e1;
    IDIWF_CUDA_CHECK(cudaEventCreate(&e0));
    IDIWF_CUDA_CHECK(cudaEventCreate(&e1));
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0, stream);
        switch (kind) {
            case 0: mb_mufu<<<blocks, threads, 0, stream>>>((float *)scratch, 0.5f); break;
            case 1: mb_dfma<<<blocks, threads, 0, stream>>>((double *)scratch, 0.5); break;
            case 2: mb_ffma<<<blocks, threads, 0, stream>>>((float *)scratch, 0.5f); break;
            default: mb_ffma2<<<blocks, threads, 0, stream>>>((float *)scratch, 0.5f); break;
        }
        cudaEventRecord(e1, stream);
        IDIWF_CUDA_CHECK(cudaEventSynchronize(e1));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    IDIWF_CUDA_CHECK(cudaGetLastError());
    const double nthreads = (double)threads * blocks;
    double ops;
    switch (kind) {
        case 0: ops = nthreads * kMbIters * 8.0; break;        // 4 sincos = 8 MUFU ops
        case 1: ops = nthreads * kMbIters * 8.0 * 2.0; break;  // 8 DFMA, 2 flop each
        case 2: ops = nthreads * kMbIters * 8.0 * 2.0; break;
        default: ops = nthreads * kMbIters * 16.0 * 2.0; break; // 8 FFMA2 = 16 FMA
    }
    *rate = ops / (best * 1e-3);
    return IDIWF_OK;
}
