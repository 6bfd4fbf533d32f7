// Counter-based random streams shared by the device samplers (sm_100a).
#pragma once

#include <stdint.h>

namespace idiwf {

// ---------------------------------------------------------------------------
// Philox4x64-10 (Salmon et al., SC 2011), numpy.random.Philox counter
// convention: the counter word 0 is incremented before each block.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void philox4x64(uint64_t c0, uint64_t c1, uint64_t c2, uint64_t c3, uint64_t k0,
                                           uint64_t k1, uint64_t &r0, uint64_t &r1, uint64_t &r2, uint64_t &r3) {
    constexpr uint64_t kM0 = 0xD2E7470EE14C6C93ull, kM1 = 0xCA5A826395121157ull;
    constexpr uint64_t kW0 = 0x9E3779B97F4A7C15ull, kW1 = 0xBB67AE8584CAA73Bull;
#pragma unroll
    for (int round = 0; round < 10; ++round) {
        const uint64_t hi0 = __umul64hi(kM0, c0), lo0 = kM0 * c0;
        const uint64_t hi1 = __umul64hi(kM1, c2), lo1 = kM1 * c2;
        const uint64_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += kW0;
        k1 += kW1;
    }
    r0 = c0;
    r1 = c1;
    r2 = c2;
    r3 = c3;
}

__device__ __forceinline__ double u01(uint64_t x) { return (double)(x >> 11) * 0x1p-53; }

// Sequential stream of uniform doubles, counter (j, c1, c2, c3), j = 1, 2, ...
struct PhiloxStream {
    uint64_t c1, c2, c3, k0, k1, j;
    uint64_t b0, b1, b2, b3;
    int pos;
    __device__ PhiloxStream(uint64_t c1_, uint64_t c2_, uint64_t c3_, uint64_t k0_, uint64_t k1_)
        : c1(c1_), c2(c2_), c3(c3_), k0(k0_), k1(k1_), j(0), b0(0), b1(0), b2(0), b3(0), pos(4) {}
    __device__ __forceinline__ double uniform() {
        if (pos == 4) {
            ++j;
            philox4x64(j, c1, c2, c3, k0, k1, b0, b1, b2, b3);
            pos = 0;
        }
        const uint64_t x = pos == 0 ? b0 : (pos == 1 ? b1 : (pos == 2 ? b2 : b3));
        ++pos;
        return u01(x);
    }
};

// Box-Muller (1958): a standard normal from two uniforms in [0, 1).
__device__ __forceinline__ double box_muller(double ua, double ub) {
    return sqrt(-2.0 * log(1.0 - ua)) * cospi(2.0 * ub);
}

// Both normals of one Box-Muller pair.
__device__ __forceinline__ void box_muller2(double ua, double ub, double &z0, double &z1) {
    const double rad = sqrt(-2.0 * log(1.0 - ua));
    double s, c;
    sincospi(2.0 * ub, &s, &c);
    z0 = rad * c;
    z1 = rad * s;
}

}  // namespace idiwf
