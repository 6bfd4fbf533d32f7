// Time-dependent direct sum for sm_100a (FP64).
//
// Per pixel p (reference: idi/simulation/time.py:48-98, simtime.cu:50-148):
//   t_j   = -s_j / c + t0_j          s_j = (d/|d| - zhat) . r_j   (far field)
//   a_j   = exp(-i (s_j k - psi_j)) [ / |d| ]
//   sort (t_j, a_j) by t_j
//   x_0 = a_0,  x_m = a_m + exp(-(t_m - t_{m-1})/tau) x_{m-1}
//   I_p = sum_{m<n-1} -tau/2 |x_m|^2 expm1(-2 (t_{m+1}-t_m)/tau) + tau/2 |x_{n-1}|^2
//
// One CTA (512 threads) handles one pixel at a time; CTAs take chunks of
// consecutive pixels from an atomic queue and walk each chunk in serpentine
// order (row by row, every other row backwards), so consecutive pixels of a
// CTA are detector neighbours.  Arrival times are computed in FP64 with the
// exact rounding sequence of the reference (np.inner as
// fma(q2,z,fma(q1,y,q0*x)), IEEE division by c), so the keys -- and therefore
// the sorted order -- are bit for bit those of the reference.
//
// Sorting.  Between neighbouring pixels the keys move by far less than their
// spacing (the arrival-time spread of the emission times dominates the
// geometric term), so the previous pixel's order is almost the new one.  The
// kernel keeps the order in shared memory as position-ordered arrays of keys
// (FP64) and 16-bit emitter indices, recomputes the keys in that order, and
// repairs it with insertion sorts over windows of 40 positions, alternating
// between two window grids offset by 20 until every window boundary is in
// order (an exact check: each window is sorted, so the whole array is sorted
// exactly when every boundary pair is).  After a bounded number of window
// passes -- and for a CTA's first pixel -- the exact full sort runs: 8192
// buckets by a monotone FP64 map of the key (so bucket order is key order),
// insertion sort inside each bucket by (key, emitter index), and an on-chip
// LSD radix sort (8 passes of 8 bits, per-warp ranking with __match_any_sync)
// if a bucket overflows.  Every path sorts by (key, emitter index), so the
// order does not depend on which one ran.
//
// The decaying scan is one pass: each thread keeps its run of 40 positions as
// an affine map x -> D x + B plus three sums from which the run's share of the
// interval integral follows once the block scan delivers the entering x.

#include <algorithm>
#include <cmath>

#include "idiwf_internal.cuh"

namespace idiwf {

constexpr int kTimeThreads = 512;
constexpr int kTimeWarps = kTimeThreads / 32;
constexpr int kTimeIPT = 40;                                 // items per thread
constexpr int kTimeMaxN = kTimeThreads * kTimeIPT;           // 20480
constexpr int kCoarse = 1024;                                 // coarse bins of the bucket map
// Slots of the position-ordered index array: one pad slot after every 80
// positions, so that the 40-position runs of a warp's threads start in
// different banks when every thread walks its own run.
constexpr int kSlotGroup = 2 * kTimeIPT;
constexpr int kTimeSlots = kTimeMaxN + kTimeMaxN / kSlotGroup;
__device__ __forceinline__ int slot(int m) { return m + m / kSlotGroup; }
constexpr size_t kTimeSmem = (size_t)kTimeMaxN * 8           // key table (by emitter index)
                             + (size_t)kTimeSlots * 2        // emitter index per sorted position
                             + (size_t)kTimeWarps * 256 * 4  // per-warp digit counters
                             + 256 * 4 + 1024                // digit bases + scan scratch
                             + (kCoarse + 4) * 4;            // first fine bucket per coarse bin
static_assert(kTimeSmem + 256 <= 232448, "time kernel shared memory above the per-block limit");
// Window passes tried on the previous pixel's order before the full sort.
constexpr int kWarmPasses = 8;
// Failed warm starts in a row after which a CTA stops trying them.
constexpr int kWarmMaxFails = 3;
// Key of the padding positions n..kTimeMaxN-1 in a full sort: the positive NaN
// with the largest payload, whose order-preserving image is the largest of all
// 64-bit patterns, so the radix sort leaves the padding behind every real key
// (NaN keys included) and positions below n always hold real emitters.
constexpr long long kPadKeyBits = 0x7FFFFFFFFFFFFFFFll;

__device__ __forceinline__ uint64_t sortable(double v) {
    const uint64_t b = (uint64_t)__double_as_longlong(v);
    return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

// Order digest base: H = sum_m (j_m + 1) B^m mod 2^64 over the sorted emitter
// indices j_m.  B = 1 mod 4, so B^d - 1 has at most 2 + log2(d) factors of 2
// and swapping two indices (differing by less than 2^15, at positions less
// than 2^15 apart) always changes H.
constexpr uint64_t kDigestBase = 0x9E3779B97F4A7C15ull;
__device__ __forceinline__ uint64_t digest_pow(int e) {
    uint64_t r = 1, b = kDigestBase;
    while (e) {
        if (e & 1) r *= b;
        b *= b;
        e >>= 1;
    }
    return r;
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

// Correctly rounded quotient a / c from ic = RN(1 / c): q0 = RN(a ic) is a
// faithful quotient, r = a - c q0 is exact in one FMA, and RN(q0 + r ic) is
// RN(a / c) (Markstein's theorem: P. Markstein, IBM J. Res. Dev. 34(1), 1990;
// Muller et al., Handbook of Floating-Point Arithmetic, the theorem on
// FMA-based correction of a faithful quotient).  The theorem needs normal
// numbers away from underflow and overflow: quotients outside [2^-960, 2^1000]
// in magnitude -- zeros, infinities and NaN included -- take the IEEE division
// (which keeps a zero's sign and an infinity).  Bit-exact against the division
// (the arrival keys must be the reference's bits).
__device__ __forceinline__ double div_rn(double a, double c, double ic) {
    const double q0 = __dmul_rn(a, ic);
    if (!(fabs(q0) >= 0x1p-960 && fabs(q0) <= 0x1p1000)) return __ddiv_rn(a, c);
    const double r = __fma_rn(-c, q0, a);
    return __fma_rn(r, ic, q0);
}

// MK: divide by c with div_rn (the on-chip kernel) or the library division (the
// large-count kernel, whose 64 registers the inlined correction would spill);
// both give the correctly rounded quotient.
// One 32-byte emitter row (x, y, z, phase) in a single 256-bit load; the
// rows are 32-byte aligned (the entry points require it of the emitter array).
__device__ __forceinline__ double4 ld_row(const double4 *p) {
    double4 r;
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w) : "l"(p));
    return r;
}

template <bool NF, bool SCALE, bool MK = true>
__device__ __forceinline__ void arrival(const GeomParams &g, double dx, double dy, double dz, double dn,
                                        double q0, double q1, double q2, const double4 &a, double t0,
                                        double c, double ic, double &t, double &s_out, double &dist_out) {
    if (!NF) {
        const double s = __fma_rn(q2, a.z, __fma_rn(q1, a.y, __dmul_rn(q0, a.x)));
        t = __dadd_rn(MK ? div_rn(-s, c, ic) : __ddiv_rn(-s, c), t0);
        s_out = s;
        dist_out = dn;
    } else {
        const double ax = __dsub_rn(dx, a.x), ay = __dsub_rn(dy, a.y), az = __dsub_rn(dz, a.z);
        const double dist = __dsqrt_rn(__fma_rn(az, az, __fma_rn(ax, ax, __dmul_rn(ay, ay))));
        const double s = __dadd_rn(__dsub_rn(dist, dn), a.z);
        t = __dadd_rn(MK ? div_rn(s, c, ic) : __ddiv_rn(s, c), t0);
        s_out = s;
        dist_out = dist;
    }
}

// Path difference s (and the 1/r distance) of one emitter, as arrival() but
// without forming the arrival time (the scan reads times from the key table).
template <bool NF>
__device__ __forceinline__ void path_only(double dx, double dy, double dz, double dn, double q0, double q1,
                                          double q2, const double4 &a, double &s_out, double &dist_out) {
    if (!NF) {
        s_out = __fma_rn(q2, a.z, __fma_rn(q1, a.y, __dmul_rn(q0, a.x)));
        dist_out = dn;
    } else {
        const double ax = __dsub_rn(dx, a.x), ay = __dsub_rn(dy, a.y), az = __dsub_rn(dz, a.z);
        const double dist = __dsqrt_rn(__fma_rn(az, az, __fma_rn(ax, ax, __dmul_rn(ay, ay))));
        s_out = __dadd_rn(__dsub_rn(dist, dn), a.z);
        dist_out = dist;
    }
}

// expm1(-x), x >= 0, for the scan.  The arguments are gaps between
// neighbouring arrival times over tau, almost always far below 1: up to 2^-4
// a Taylor polynomial of degree 10 in Horner form (coefficients 1/k!) is exact
// to FP64 rounding (the first omitted term is below 3e-19 of the result);
// larger arguments use the library function.  (The on-chip kernel uses it; in
// the 64-register large-count kernel the inlined polynomial measured slower
// than the library calls.)  The coefficient tables of this file live in
// constant memory: an FP64 FMA takes a constant-bank operand directly, where a
// 64-bit literal costs two moves into registers (measured: half the
// instructions of the polynomials).
__constant__ double kInvFact[11] = {1.0,       1.0,        1.0 / 2,     1.0 / 6,      1.0 / 24,      1.0 / 120,
                                    1.0 / 720, 1.0 / 5040, 1.0 / 40320, 1.0 / 362880, 1.0 / 3628800};
__device__ __forceinline__ double expm1_neg(double x) {
    if (!(x <= 0.0625)) return expm1(-x);
    const double t = -x;
    double q = kInvFact[10];
#pragma unroll
    for (int k = 9; k >= 1; --k) q = __fma_rn(q, t, kInvFact[k]);
    return t * q;  // t (1 + t/2! + ... + t^9/10!)
}

// sin and cos of x (FP64), for the time path's amplitudes.  Cody-Waite
// reduction (W. J. Cody and W. Waite, Software Manual for the Elementary
// Functions, 1980): n = rint(x 2/pi), a = (x - n P1) - n P2 with P1 + P2 = pi/2
// to twice the precision (P1 = RN(pi/2), P2 = RN(pi/2 - P1)), |a| <= pi/4 up
// to rounding, good to ~1e-16 rad for |x| far below 2^40; then the Taylor
// series of sin and cos (coefficients (-1)^k / k!) to degrees 17 and 18, whose
// first omitted terms are below 1e-19 on |a| <= pi/4, in Horner form over a^2;
// the quadrant n mod 4 swaps and negates.  Arguments beyond 2^30 take the
// library function.
// Cody-Waite constants {2/pi, P1, P2} and the Taylor coefficients of sin
// (degree 17 down to 3) and cos (degree 18 down to 2), highest first.
__constant__ double kCW[3] = {0.63661977236758134308, 1.5707963267948966192, 6.123233995736766036e-17};
__constant__ double kSinC[8] = {1.0 / 355687428096000.0, -1.0 / 1307674368000.0, 1.0 / 6227020800.0,
                                -1.0 / 39916800.0,       1.0 / 362880.0,         -1.0 / 5040.0,
                                1.0 / 120.0,             -1.0 / 6.0};
__constant__ double kCosC[9] = {1.0 / 6402373705728000.0, -1.0 / 20922789888000.0, 1.0 / 87178291200.0,
                                -1.0 / 479001600.0,       1.0 / 3628800.0,         -1.0 / 40320.0,
                                1.0 / 720.0,              -1.0 / 24.0,             0.5};
__device__ __forceinline__ void sincos_cw(double x, double &sn, double &cs) {
    if (!(fabs(x) <= 0x1p30)) {
        sincos(x, &sn, &cs);
        return;
    }
    const double nd = rint(x * kCW[0]);
    double a = __fma_rn(-nd, kCW[1], x);
    a = __fma_rn(-nd, kCW[2], a);
    const double a2 = a * a;
    double ps = kSinC[0];
#pragma unroll
    for (int i = 1; i < 8; ++i) ps = __fma_rn(ps, a2, kSinC[i]);
    const double s = __fma_rn(a * a2, ps, a);
    double pc = kCosC[0];
#pragma unroll
    for (int i = 1; i < 9; ++i) pc = __fma_rn(pc, a2, kCosC[i]);
    const double co = __fma_rn(-a2, pc, 1.0);
    const int q = (int)(((long long)nd) & 3);
    sn = (q & 1) ? co : s;
    cs = (q & 1) ? s : co;
    if (q == 1 || q == 2) cs = -cs;
    if (q >= 2) sn = -sn;
}

// CW: sine and cosine by sincos_cw (the on-chip kernel) or the library (the
// 64-register large-count kernel).
template <bool NF, bool SCALE, bool CW = true>
__device__ __forceinline__ void amplitude(double k, double s, double psi, double dist, double &re, double &im) {
    double th;
    if (!NF) th = -__dsub_rn(__dmul_rn(s, k), psi);  // time.py:94 exp(-1j*(s*k-phases))
    else th = __dadd_rn(__dmul_rn(s, k), psi);       // simtime.cu:71 phase = s*k + w
    double sn, cs;
    if (CW) sincos_cw(th, sn, cs);
    else sincos(th, &sn, &cs);
    if (SCALE) {
        cs = __ddiv_rn(cs, dist);
        sn = __ddiv_rn(sn, dist);
    }
    re = cs;
    im = sn;
}

// Block-wide min / max of the keys; result broadcast through smem (2 doubles).
__device__ __forceinline__ void block_minmax(double &lo, double &hi, double *sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    __syncthreads();
    if (lane == 0) {
        sm[2 * warp] = lo;
        sm[2 * warp + 1] = hi;
    }
    __syncthreads();
    lo = sm[0];
    hi = sm[1];
    for (int w = 1; w < kTimeWarps; ++w) {
        lo = fmin(lo, sm[2 * w]);
        hi = fmax(hi, sm[2 * w + 1]);
    }
    __syncthreads();
}

// Exact sort of emitter indices by key, by buckets.  The bucket of a key is
// a non-decreasing function of the key in IEEE arithmetic, so bucket order is
// key order; each bucket is then insertion-sorted by (key, emitter index).
// The map has two levels so that buckets hold about the same number of keys
// whatever the keys' distribution (arrival times are near-Gaussian, and a
// linear map crowds the middle buckets, whose insertion sort then holds the
// whole CTA at the next barrier): u = (t - kmin) kCoarse / (kmax - kmin) picks
// coarse bin c = floor(u); coarse bin c owns the fine buckets [B_c, B_c+1),
// B_c = c + floor(P_c (kBuckets - kCoarse) / n) with P_c the keys below bin c
// (at least one bucket per coarse bin), and the key goes to fine bucket
// B_c + floor((u - c) (B_c+1 - B_c)), clamped into the bin's range.  Every step
// is monotone in t.  Returns false (perm undefined) when a bucket holds more
// than kMaxBucket keys; the caller then runs the radix sort.  cnt: kBuckets/2
// words of packed 16-bit counters; coarse: kCoarse + 1 words.
constexpr int kBuckets = 8192;
constexpr int kMaxBucket = 128;
constexpr int kBucketsPerThread = kBuckets / kTimeThreads;  // 16
constexpr int kCoarsePerThread = kCoarse / kTimeThreads;    // 2

__device__ __forceinline__ int coarse_of(double u) { return min(max(__double2int_rz(u), 0), kCoarse - 1); }

__device__ __forceinline__ uint32_t fine_bucket(double t, double kmin, double scale, const uint32_t *coarse) {
    const double u = __dmul_rn(__dsub_rn(t, kmin), scale);
    const int c = coarse_of(u);
    const uint32_t b0 = coarse[c], nb = coarse[c + 1] - b0;
    const int f = __double2int_rz(__dmul_rn(__dsub_rn(u, (double)c), (double)nb));
    return b0 + (uint32_t)min(max(f, 0), (int)nb - 1);
}
__device__ __forceinline__ uint32_t cnt_get(const uint32_t *cnt, uint32_t b) {
    const uint32_t w = cnt[b >> 1];
    return (b & 1) ? (w >> 16) : (w & 0xFFFFu);
}

__device__ bool bucket_sort(const double *keytab, uint16_t *perm, uint32_t *cnt, uint32_t *coarse, int n,
                            double kmin, double kmax, double *scratch, int *s_flag) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (!(kmax > kmin)) {
        // all keys equal (or one key): stable order is emitter order
        for (int m = tid; m < n; m += kTimeThreads) perm[m] = (uint16_t)m;
        __syncthreads();
        return true;
    }
    const double scale = (double)kCoarse / (kmax - kmin);
    for (int w = tid; w < kBuckets / 2; w += kTimeThreads) cnt[w] = 0u;
    for (int c = tid; c <= kCoarse; c += kTimeThreads) coarse[c] = 0u;
    if (tid == 0) *s_flag = 0;
    __syncthreads();
    for (int j = tid; j < n; j += kTimeThreads)
        atomicAdd(&coarse[coarse_of(__dmul_rn(__dsub_rn(keytab[j], kmin), scale))], 1u);
    __syncthreads();
    uint32_t *wsum = reinterpret_cast<uint32_t *>(scratch);  // 16 words
    {
        // B_c from the exclusive prefix of the coarse counts; thread t owns bins [2t, 2t+2)
        uint32_t cc[kCoarsePerThread], sum = 0;
#pragma unroll
        for (int i = 0; i < kCoarsePerThread; ++i) {
            cc[i] = coarse[tid * kCoarsePerThread + i];
            sum += cc[i];
        }
        uint32_t incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        uint32_t pre = incl - sum;
        for (int w = 0; w < warp; ++w) pre += wsum[w];
        __syncthreads();
#pragma unroll
        for (int i = 0; i < kCoarsePerThread; ++i) {
            const int c = tid * kCoarsePerThread + i;
            coarse[c] = (uint32_t)c + (uint32_t)(((uint64_t)pre * (kBuckets - kCoarse)) / (uint64_t)n);
            pre += cc[i];
        }
        if (tid == kTimeThreads - 1) coarse[kCoarse] = kBuckets;
    }
    __syncthreads();
    // the fine bucket of each of the thread's keys, two 13-bit ids per word,
    // kept for the scatter
    uint32_t fb[kTimeIPT / 2];
#pragma unroll
    for (int i = 0; i < kTimeIPT; ++i) {
        const int j = tid + i * kTimeThreads;
        uint32_t b = 0;
        if (j < n) {
            b = fine_bucket(keytab[j], kmin, scale, coarse);
            atomicAdd(&cnt[b >> 1], (b & 1) ? 0x10000u : 1u);
        }
        if (i & 1) fb[i / 2] |= b << 16;
        else fb[i / 2] = b;
    }
    __syncthreads();
    // exclusive scan of the counters: thread t owns buckets [16t, 16t+16)
    uint32_t loc[kBucketsPerThread];
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < kBucketsPerThread; ++i) {
        loc[i] = cnt_get(cnt, tid * kBucketsPerThread + i);
        sum += loc[i];
    }
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    uint32_t run = incl - sum;
    for (int w = 0; w < warp; ++w) run += wsum[w];
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kBucketsPerThread; i += 2) {
        const uint32_t s0 = run, s1 = run + loc[i];
        cnt[(tid * kBucketsPerThread + i) >> 1] = s0 | (s1 << 16);
        if (loc[i] > kMaxBucket || loc[i + 1] > kMaxBucket) *s_flag = 1;
        run = s1 + loc[i + 1];
    }
    __syncthreads();
    if (*s_flag) return false;  // uniform: every thread read the same flag after the barrier
    // scatter: afterwards cnt holds the end (= next start) of every bucket
#pragma unroll
    for (int i = 0; i < kTimeIPT; ++i) {
        const int j = tid + i * kTimeThreads;
        if (j < n) {
            const uint32_t b = (i & 1) ? (fb[i / 2] >> 16) : (fb[i / 2] & 0xFFFFu);
            const uint32_t old = atomicAdd(&cnt[b >> 1], (b & 1) ? 0x10000u : 1u);
            perm[(b & 1) ? (old >> 16) : (old & 0xFFFFu)] = (uint16_t)j;
        }
    }

    __syncthreads();
    // insertion sort inside each bucket by (key, emitter index)
    for (int i = 0; i < kBucketsPerThread; ++i) {
        const uint32_t b = tid * kBucketsPerThread + i;
        const int start = b == 0 ? 0 : (int)cnt_get(cnt, b - 1);
        const int end = (int)cnt_get(cnt, b);
        for (int m = start + 1; m < end; ++m) {
            const uint16_t v = perm[m];
            const double kv = keytab[v];
            int q = m - 1;
            while (q >= start) {
                const uint16_t u = perm[q];
                const double ku = keytab[u];
                if (ku < kv || (ku == kv && u < v)) break;
                perm[q + 1] = u;
                --q;
            }
            perm[q + 1] = v;
        }
    }
    __syncthreads();
    return true;
}

// Stable LSD radix sort (8 passes of 8 bits) of emitter indices by the
// order-preserving 64-bit image of their keys; the fallback of bucket_sort.
// Keys of positions >= n are +inf and stay at the end.
__device__ void radix_sort(const double *keytab, uint16_t *perm, uint32_t *H, uint32_t *base) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int S = 32 * kTimeIPT;
    const uint32_t lt_mask = (1u << lane) - 1u;
    uint16_t idx[kTimeIPT];
#pragma unroll
    for (int i = 0; i < kTimeIPT; ++i) idx[i] = (uint16_t)(warp * S + i * 32 + lane);
    __syncthreads();
    for (int pass = 0; pass < 8; ++pass) {
        const int shift = pass * 8;
        uint32_t *Hw = H + warp * 256;
        for (int k = lane; k < 256; k += 32) Hw[k] = 0;
        __syncwarp();
        for (int i = 0; i < kTimeIPT; ++i) {
            const uint32_t dg = (uint32_t)(sortable(keytab[idx[i]]) >> shift) & 255u;
            const uint32_t peers = __match_any_sync(0xffffffffu, dg);
            if ((peers & lt_mask) == 0) Hw[dg] += __popc(peers);
            __syncwarp();
        }
        __syncthreads();
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
}

// (key, emitter index) order; false both ways for an unordered (NaN) key,
// which then never passes the boundary check and takes the full sort.
__device__ __forceinline__ bool before(double ka, int ja, double kb, int jb) {
    return ka < kb || (ka == kb && ja < jb);
}

// Insertion sort of positions [lo, hi) (hi - lo < kSlotGroup) of the
// position-ordered emitter indices P by (key, emitter index), keys from the
// table by emitter.  P comes from the previous pixel's order, so the inner
// loop rarely runs; (kprev, jprev) is the entry at position m - 1
// throughout, and the next position's entry is loaded one step ahead (an
// insertion only rewrites positions up to m).
__device__ __forceinline__ void window_sort(const double *keytab, uint16_t *P, int lo, int hi) {
    // slots of [lo, hi): contiguous except for one pad slot at the next
    // multiple of kSlotGroup
    const int off = lo / kSlotGroup, cut = (off + 1) * kSlotGroup;
    auto sl = [&](int m) { return m + off + (m >= cut ? 1 : 0); };
    int jprev = P[sl(lo)];
    double kprev = keytab[jprev];
    int v = lo + 1 < hi ? P[sl(lo + 1)] : 0;
    double kv = keytab[v];
    for (int m = lo + 1; m < hi; ++m) {
        const int vn = m + 1 < hi ? P[sl(m + 1)] : 0;
        const double kn = keytab[vn];
        if (before(kprev, jprev, kv, v)) {
            kprev = kv;
            jprev = v;
        } else {
            // shift the entries behind v up by one
            int q = m - 1;
            P[sl(m)] = (uint16_t)jprev;
            while (--q >= lo) {
                const int u = P[sl(q)];
                if (before(keytab[u], u, kv, v)) break;
                P[sl(q + 1)] = (uint16_t)u;
            }
            P[sl(q + 1)] = (uint16_t)v;
            // position m now holds (kprev, jprev)
        }
        v = vn;
        kv = kn;
    }
}

template <bool NF, bool SCALE, bool DIGEST>
__global__ void __launch_bounds__(kTimeThreads, 1) time_kernel(const GeomParams g, const double *__restrict__ atoms,
                                                                const double *__restrict__ times, int n, double c,
                                                                double tau, double *__restrict__ out,
                                                                WsHeader *__restrict__ hdr, int order_pixel,
                                                                int *__restrict__ order_out,
                                                                double *__restrict__ keys_out,
                                                                uint64_t *__restrict__ digest, int chunk) {
    extern __shared__ __align__(16) unsigned char smem[];
    double *keytab = reinterpret_cast<double *>(smem);
    uint16_t *P = reinterpret_cast<uint16_t *>(smem + (size_t)kTimeMaxN * 8);
    uint32_t *H = reinterpret_cast<uint32_t *>(smem + (size_t)kTimeMaxN * 8 + (size_t)kTimeSlots * 2);
    uint32_t *base = H + kTimeWarps * 256;
    double *scratch = reinterpret_cast<double *>(base + 256);  // 128 doubles
    uint32_t *coarse = reinterpret_cast<uint32_t *>(scratch + 128);
    __shared__ uint64_t s_dig[kTimeWarps];
    __shared__ int s_pix, s_flag;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int npix = g.nx * g.ny;
    const double ic = 1.0 / c;  // correctly rounded (IEEE division)
    const double4 *atoms4 = reinterpret_cast<const double4 *>(atoms);
    // the scan's exponents use a multiply by 1/tau (1 ulp from the reference's
    // division, ~1e-16 relative in the decay); only the sort keys must match bit for bit
    const double inv_tau = 1.0 / tau;

    // CTA-uniform sort state: whether (K, P) hold the previous pixel's order,
    // and whether warm starts are still tried
    bool have = false;
    int fails = 0;
    // order_pixel >= 0: process that one pixel only, record its sorted order
    // and write its intensity to out[0]
    int iter = 0;
    for (;;) {
        __syncthreads();
        if (tid == 0)
            s_pix = order_pixel >= 0 ? (iter == 0 ? 0 : npix) : (int)atomicAdd(&hdr->work_counter, (unsigned)chunk);
        __syncthreads();
        ++iter;
        const int c0 = s_pix;
        if (c0 >= npix) break;
        const int c1 = order_pixel >= 0 ? c0 + 1 : min(c0 + chunk, npix);
        for (int pl = c0; pl < c1; ++pl) {
            int ix, iy;
            if (order_pixel >= 0) {
                ix = order_pixel / g.ny;
                iy = order_pixel - ix * g.ny;
            } else {
                // serpentine walk: odd rows backwards
                ix = pl / g.ny;
                const int r = pl - ix * g.ny;
                iy = (ix & 1) ? g.ny - 1 - r : r;
            }
            const int p = ix * g.ny + iy;
            double dx, dy, dz;
            pixel_time(g, ix, iy, dx, dy, dz);
            // time.py:89-91 (np.linalg.norm = sqrt((x*x + y*y) + z*z); q = det/d; q_z -= 1)
            const double dn =
                __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
            const double q0 = __ddiv_rn(dx, dn), q1 = __ddiv_rn(dy, dn), q2 = __dsub_rn(__ddiv_rn(dz, dn), 1.0);

            // ---- keys: table by emitter index (coalesced), padding last ----
            // (the rows of KB emitters per thread are loaded before any is used)
            double kmin = __longlong_as_double(0x7FF0000000000000ll), kmax = -kmin;
            {
                constexpr int KB = NF ? 4 : 8;
#pragma unroll 1
                for (int b = 0; b < kTimeIPT; b += KB) {
                    double4 aa[KB];
                    double tt[KB];
#pragma unroll
                    for (int u = 0; u < KB; ++u) {
                        const int j = tid + (b + u) * kTimeThreads;
                        aa[u] = j < n ? ld_row(atoms4 + j) : make_double4(0.0, 0.0, 0.0, 0.0);
                        tt[u] = j < n ? times[j] : 0.0;
                    }
                    if (!NF) {
                        // far field without branches: the Markstein quotient of every
                        // row, and the IEEE division after the batch for a quotient out of
                        // div_rn's range (a zero path difference, say); the padding keys
                        // (a NaN) leave min and max alone
                        double tq[KB];
                        bool redo = false;
#pragma unroll
                        for (int u = 0; u < KB; ++u) {
                            const double sp = __fma_rn(q2, aa[u].z, __fma_rn(q1, aa[u].y, __dmul_rn(q0, aa[u].x)));
                            const double qa = __dmul_rn(-sp, ic);
                            tq[u] = __fma_rn(__fma_rn(-c, qa, -sp), ic, qa);
                            redo |= tid + (b + u) * kTimeThreads < n && !(fabs(qa) >= 0x1p-960 && fabs(qa) <= 0x1p1000);
                        }
                        if (redo) {
#pragma unroll
                            for (int u = 0; u < KB; ++u) {
                                const double sp =
                                    __fma_rn(q2, aa[u].z, __fma_rn(q1, aa[u].y, __dmul_rn(q0, aa[u].x)));
                                tq[u] = div_rn(-sp, c, ic);
                            }
                        }
#pragma unroll
                        for (int u = 0; u < KB; ++u) {
                            const int j = tid + (b + u) * kTimeThreads;
                            const double t = j < n ? __dadd_rn(tq[u], tt[u]) : __longlong_as_double(kPadKeyBits);
                            kmin = fmin(kmin, t);
                            kmax = fmax(kmax, t);
                            keytab[j] = t;
                        }
                    } else {
#pragma unroll
                        for (int u = 0; u < KB; ++u) {
                            const int j = tid + (b + u) * kTimeThreads;
                            double t = __longlong_as_double(kPadKeyBits);
                            if (j < n) {
                                double s, dist;
                                arrival<NF, SCALE>(g, dx, dy, dz, dn, q0, q1, q2, aa[u], tt[u], c, ic, t, s, dist);
                                kmin = fmin(kmin, t);
                                kmax = fmax(kmax, t);
                            }
                            keytab[j] = t;
                        }
                    }
                }
            }
            __syncthreads();

            // ---- sort: warm start from the previous pixel's order ----
            bool sorted = false;
            if (have && fails < kWarmMaxFails) {
                // thread t's window: [40t, 40t+40) on even passes, [40t-20, 40t+20) on odd
                // ones (the last thread's odd window runs to the end).  After a pass every
                // window is sorted, so a window of the other grid -- two sorted halves --
                // is out of order only if the boundary at its middle is: a thread sorts its
                // window in the first pass, and later only when that boundary was found out
                // of order (dirty).  The boundary a thread checks is the middle of its next
                // window; together the threads check every boundary of the pass's grid.
                bool dirty = true;
                for (int pass = 0; pass < kWarmPasses; ++pass) {
                    const int sh = (pass & 1) ? kTimeIPT / 2 : 0;
                    const int lo = max(tid * kTimeIPT - sh, 0);
                    const int hi = min(tid == kTimeThreads - 1 ? kTimeMaxN : (tid + 1) * kTimeIPT - sh, n);
                    // (the previous pass's __syncthreads_or ordered its reads before these writes)
                    if (dirty && lo < hi) window_sort(keytab, P, lo, hi);
                    __syncthreads();
                    const int b = (pass & 1) ? (tid + 1) * kTimeIPT - sh : tid * kTimeIPT;
                    bool bad = false;
                    if (b >= 1 && b < n) {
                        const int u = P[slot(b - 1)], v = P[slot(b)];
                        bad = !before(keytab[u], u, keytab[v], v);
                    }
                    dirty = bad;
                    if (!__syncthreads_or(bad)) {
                        sorted = true;
                        break;
                    }
                    if (pass == 0) {
                        // Between neighbouring pixels the few pairs still out of order sit
                        // at even boundaries and have moved by a position or two: first a
                        // window of 2 kPatch positions around each such boundary.  Only
                        // the pairs at those windows' ends can then be out of order; where
                        // one is, the odd window around it (which holds the short one)
                        // takes over in the next pass.
                        constexpr int kPatch = 8;
                        const int plo = max(b - kPatch, 0), phi = min(b + kPatch, n);
                        if (bad) window_sort(keytab, P, plo, phi);
                        __syncthreads();
                        bool pbad = false;
                        if (bad) {
                            if (plo >= 1) {
                                const int u = P[slot(plo - 1)], v = P[slot(plo)];
                                pbad = !before(keytab[u], u, keytab[v], v);
                            }
                            if (phi < n) {
                                const int u = P[slot(phi - 1)], v = P[slot(phi)];
                                pbad = pbad || !before(keytab[u], u, keytab[v], v);
                            }
                        }
                        dirty = pbad;
                        if (!__syncthreads_or(pbad)) {
                            sorted = true;
                            break;
                        }
                    }
                }
                fails = sorted ? 0 : fails + 1;
                if (!sorted && tid == 0) atomicAdd(&hdr->work_counter3, 1u);  // warm starts given up
            }
            if (!sorted) {
                // ---- full sort ----
                if (tid == 0) atomicAdd(&hdr->work_counter2, 1u);  // full sorts
                block_minmax(kmin, kmax, scratch + 96);
                if (!bucket_sort(keytab, P, reinterpret_cast<uint32_t *>(H), coarse, n, kmin, kmax, scratch,
                                 &s_flag)) {
                    radix_sort(keytab, P, H, base);
                }
                // P[m] (unpadded) = emitter at sorted position m: move to slots
                uint32_t pk[kTimeIPT / 2];
                const int m0 = tid * kTimeIPT;
#pragma unroll
                for (int i = 0; i < kTimeIPT / 2; ++i)
                    pk[i] = (uint32_t)P[m0 + 2 * i] | ((uint32_t)P[m0 + 2 * i + 1] << 16);
                __syncthreads();
#pragma unroll
                for (int i = 0; i < kTimeIPT / 2; ++i) {
                    P[slot(m0) + 2 * i] = (uint16_t)(pk[i] & 0xFFFFu);
                    P[slot(m0) + 2 * i + 1] = (uint16_t)(pk[i] >> 16);
                }
                __syncthreads();
            }
            have = true;
            // P[slot(m)]: emitter at sorted position m < n

            if (order_pixel >= 0) {
                for (int m = tid; m < n; m += kTimeThreads) {
                    order_out[m] = P[slot(m)];
                    keys_out[m] = keytab[P[slot(m)]];
                }
            }

            // ---- decaying scan over the sorted sequence, one pass ----
            // Thread t owns positions [40t, 40t+40).  Inside its run
            //   x_m = D_m X + B_m,  D_m = prod of the run's decays up to m,
            // with X the value entering the run (known only after the block scan),
            // so sum_m w_m |x_m|^2 = |X|^2 S1 + 2 Re(X conj(S2)) + S3 with
            //   S1 = sum w D^2, S2 = sum w D B, S3 = sum w |B|^2
            // and w_m = -tau/2 expm1(-2 (t_{m+1} - t_m)/tau), w_{n-1} = tau/2
            // (the interval integral of time.py:36-45).  Each gap g enters twice:
            // as the decay exp(-g/tau) = 1 + em of the later position and as the
            // weight -tau/2 expm1(-2 g/tau) = -tau/2 em (2 + em) of the earlier one,
            // with em = expm1(-g/tau): one polynomial per gap, no cancellation.
            const int m0 = tid * kTimeIPT;
            const uint16_t *Pr = P + slot(m0);  // the run's slots are contiguous
            double Dm = 1.0, Br = 0.0, Bi = 0.0;
            double S1 = 0.0, S2r = 0.0, S2i = 0.0, S3 = 0.0;
            uint64_t h = 0, pw = DIGEST && m0 < n ? digest_pow(m0) : 0;
            // the neighbours' keys travel in registers from one position to the
            // next, and the emitter rows are loaded two positions ahead
            int j_next = 0;
            double t_next = 0.0, em_in = 0.0;
            double4 a_next = make_double4(0.0, 0.0, 0.0, 0.0), a_next2 = a_next;
            if (m0 < n) {
                j_next = Pr[0];
                t_next = keytab[j_next];
                a_next = ld_row(atoms4 + j_next);
                if (m0 + 1 < n) a_next2 = ld_row(atoms4 + Pr[1]);
                if (m0 > 0) em_in = expm1_neg(__dsub_rn(t_next, keytab[P[slot(m0 - 1)]]) * inv_tau);
            }
            for (int i = 0; i < kTimeIPT; ++i) {
                const int m = m0 + i;
                if (m >= n) break;
                const double tj = t_next;
                const double4 a = a_next;
                a_next = a_next2;
                if (DIGEST) {
                    h += (uint64_t)(j_next + 1) * pw;
                    pw *= kDigestBase;
                }
                if (m + 1 < n) {
                    j_next = i + 1 < kTimeIPT ? Pr[i + 1] : P[slot(m + 1)];
                    t_next = keytab[j_next];
                }
                if (i + 2 < kTimeIPT && m + 2 < n) a_next2 = ld_row(atoms4 + Pr[i + 2]);
                double s, dist, re, im;
                path_only<NF>(dx, dy, dz, dn, q0, q1, q2, a, s, dist);
                amplitude<NF, SCALE>(g.k, s, a.w, dist, re, im);
                const double dec = m == 0 ? 0.0 : 1.0 + em_in;
                Dm *= dec;
                Br = fma(dec, Br, re);
                Bi = fma(dec, Bi, im);
                double w = tau / 2;
                if (m < n - 1) {
                    em_in = expm1_neg(__dsub_rn(t_next, tj) * inv_tau);
                    w = (-tau / 2) * (em_in * (2.0 + em_in));
                }
                const double wD = w * Dm;
                S1 = fma(wD, Dm, S1);
                S2r = fma(wD, Br, S2r);
                S2i = fma(wD, Bi, S2i);
                S3 = fma(w, fma(Br, Br, Bi * Bi), S3);
            }
            const Affine agg = {Dm, Br, Bi};
            // block exclusive scan of the run maps
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
            // X entering this thread's run = excl applied to x_{-1} = 0
            const double Xr = excl.br, Xi = excl.bi;
            double part = fma(fma(Xr, Xr, Xi * Xi), S1, fma(2.0, fma(Xr, S2r, Xi * S2i), S3));
            // block sum (and of the order digest)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                part += __shfl_down_sync(0xffffffffu, part, o);
                if (DIGEST) h += __shfl_down_sync(0xffffffffu, h, o);
            }
            __syncthreads();
            if (lane == 0) {
                scratch[64 + warp] = part;
                if (DIGEST) s_dig[warp] = h;
            }
            __syncthreads();
            if (tid == 0) {
                double tot = 0.0;
                uint64_t hh = 0;
                for (int w = 0; w < kTimeWarps; ++w) {
                    tot += scratch[64 + w];
                    if (DIGEST) hh += s_dig[w];
                }
                out[order_pixel >= 0 ? 0 : p] = tot;
                if (DIGEST && order_pixel < 0) digest[p] = hh;
            }
            // the next pixel's key pass overwrites the key table and P, which the scan reads
            // across runs, and scratch, which thread 0 has just read
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------
// Large emitter counts (n > kTimeMaxN): the same algorithm with the per-pixel
// arrays in a global workspace slice per CTA -- keys (FP64, by emitter),
// two int32 permutations -- and the bucket counters (uint32, up to
// kLargeBuckets) in shared memory.  Fallback for an overfull bucket: a
// stable LSD radix sort over the whole array in tiles.
// ---------------------------------------------------------------------------
constexpr int kLargeBuckets = 16384;
constexpr int kLargeMaxBucket = 256;
constexpr size_t kLargeSmem = (size_t)kLargeBuckets * 4  // also holds the radix counters
                              + (kCoarse + 4) * 4;      // first fine bucket per coarse bin

__host__ __device__ __forceinline__ int large_buckets(int64_t n) {
    int nb = 8 * kCoarse;  // n > 20480 here: at least 8192 buckets, a multiple of the threads
    while (nb < kLargeBuckets && (int64_t)nb * 4 < n) nb <<= 1;
    return nb;
}

// A CTA's slice: keys (8 B per emitter), the sorted records (16 B) and two
// index arrays for the radix fallback (4 B each).
struct SortRec {
    double key;
    int idx;
    int pad;
};
__host__ __device__ __forceinline__ size_t large_slice_bytes(int64_t n) {
    return ((size_t)n * 32 + 255) & ~(size_t)255;
}

// The two-level map of bucket_sort with nb fine buckets (nb >= 8192 here).
__device__ __forceinline__ uint32_t fine_bucket_n(double t, double kmin, double scale, const uint32_t *coarse) {
    return fine_bucket(t, kmin, scale, coarse);
}

// Sorted (key, emitter) records in rec: the scatter moves each record to its
// bucket and the insertion sort works on the bucket's contiguous records, so
// no pass gathers keys through a permutation.
__device__ bool bucket_sort_large(const double *keys, SortRec *rec, uint32_t *cnt, uint32_t *coarse, int n, int nb,
                                  double kmin, double kmax, double *scratch, int *s_flag) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (!(kmax > kmin)) {
        for (int m = tid; m < n; m += kTimeThreads) rec[m] = SortRec{keys[m], m, 0};
        __syncthreads();
        return true;
    }
    const double scale = (double)kCoarse / (kmax - kmin);
    const int per = nb / kTimeThreads;
    for (int b = tid; b < nb; b += kTimeThreads) cnt[b] = 0u;
    for (int c = tid; c <= kCoarse; c += kTimeThreads) coarse[c] = 0u;
    if (tid == 0) *s_flag = 0;
    __syncthreads();
    for (int j = tid; j < n; j += kTimeThreads)
        atomicAdd(&coarse[coarse_of(__dmul_rn(__dsub_rn(keys[j], kmin), scale))], 1u);
    __syncthreads();
    uint32_t *wsum = reinterpret_cast<uint32_t *>(scratch);
    {
        uint32_t cc[kCoarsePerThread], csum = 0;
#pragma unroll
        for (int i = 0; i < kCoarsePerThread; ++i) {
            cc[i] = coarse[tid * kCoarsePerThread + i];
            csum += cc[i];
        }
        uint32_t cincl = csum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, cincl, o);
            if (lane >= o) cincl += y;
        }
        if (lane == 31) wsum[warp] = cincl;
        __syncthreads();
        uint32_t pre = cincl - csum;
        for (int w = 0; w < warp; ++w) pre += wsum[w];
        __syncthreads();
#pragma unroll
        for (int i = 0; i < kCoarsePerThread; ++i) {
            const int c = tid * kCoarsePerThread + i;
            coarse[c] = (uint32_t)c + (uint32_t)(((uint64_t)pre * (uint64_t)(nb - kCoarse)) / (uint64_t)n);
            pre += cc[i];
        }
        if (tid == kTimeThreads - 1) coarse[kCoarse] = (uint32_t)nb;
    }
    __syncthreads();
    for (int j = tid; j < n; j += kTimeThreads) atomicAdd(&cnt[fine_bucket_n(keys[j], kmin, scale, coarse)], 1u);
    __syncthreads();
    uint32_t sum = 0, big = 0;
    for (int i = 0; i < per; ++i) {
        const uint32_t c = cnt[tid * per + i];
        sum += c;
        big |= c > kLargeMaxBucket;
    }
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    if (big) *s_flag = 1;
    __syncthreads();
    uint32_t run = incl - sum;
    for (int w = 0; w < warp; ++w) run += wsum[w];
    __syncthreads();
    for (int i = 0; i < per; ++i) {
        const uint32_t c = cnt[tid * per + i];
        cnt[tid * per + i] = run;
        run += c;
    }
    __syncthreads();
    if (*s_flag) return false;
    // scatter: afterwards cnt[b] is the end of bucket b
    for (int j = tid; j < n; j += kTimeThreads) {
        const double kj = keys[j];
        const uint32_t pos = atomicAdd(&cnt[fine_bucket_n(kj, kmin, scale, coarse)], 1u);
        rec[pos] = SortRec{kj, j, 0};
    }
    __syncthreads();
    for (int i = 0; i < per; ++i) {
        const int b = tid * per + i;
        const int start = b == 0 ? 0 : (int)cnt[b - 1];
        const int end = (int)cnt[b];
        for (int m = start + 1; m < end; ++m) {
            const SortRec v = rec[m];
            int q = m - 1;
            while (q >= start) {
                const SortRec u = rec[q];
                if (u.key < v.key || (u.key == v.key && u.idx < v.idx)) break;
                rec[q + 1] = u;
                --q;
            }
            rec[q + 1] = v;
        }
    }
    __syncthreads();
    return true;
}

// Stable LSD radix sort (8 passes of 8 bits) of emitter indices by the
// order-preserving image of their keys.  Items go through in tiles of
// kTimeThreads * kLargeIPT; inside a tile warp w takes the items
// [w S, (w+1) S), lane-interleaved, so ranks follow item order; digit bases
// carry over from tile to tile.  Result in a (the input order is built here).
constexpr int kLargeIPT = 16;

__device__ void radix_sort_large(const double *keys, int *a, int *b, int n, uint32_t *H, uint32_t *base) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int S = 32 * kLargeIPT, T = kTimeThreads * kLargeIPT;
    const uint32_t lt_mask = (1u << lane) - 1u;
    for (int m = tid; m < n; m += kTimeThreads) a[m] = m;
    __syncthreads();
    for (int pass = 0; pass < 8; ++pass) {
        const int shift = pass * 8;
        // global digit histogram -> exclusive bases
        for (int k = tid; k < 256; k += kTimeThreads) base[k] = 0;
        __syncthreads();
        for (int m = tid; m < n; m += kTimeThreads)
            atomicAdd(&base[(uint32_t)(sortable(keys[a[m]]) >> shift) & 255u], 1u);
        __syncthreads();
        if (warp == 0) {
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
        for (int t0 = 0; t0 < n; t0 += T) {
            uint32_t *Hw = H + warp * 256;
            for (int k = lane; k < 256; k += 32) Hw[k] = 0;
            __syncwarp();
            // per-warp digit counts of this tile
            for (int i = 0; i < kLargeIPT; ++i) {
                const int m = t0 + warp * S + i * 32 + lane;
                const uint32_t dg = m < n ? (uint32_t)(sortable(keys[a[m]]) >> shift) & 255u : 256u;
                const uint32_t peers = __match_any_sync(0xffffffffu, dg);
                if (dg < 256u && (peers & lt_mask) == 0) Hw[dg] += __popc(peers);
                __syncwarp();
            }
            __syncthreads();
            // warp offsets inside the tile, and the tile's totals added to the bases
            if (tid < 256) {
                uint32_t run = base[tid];
                for (int w = 0; w < kTimeWarps; ++w) {
                    const uint32_t h = H[w * 256 + tid];
                    H[w * 256 + tid] = run;
                    run += h;
                }
                base[tid] = run;
            }
            __syncthreads();
            for (int i = 0; i < kLargeIPT; ++i) {
                const int m = t0 + warp * S + i * 32 + lane;
                const int e = m < n ? a[m] : 0;
                const uint32_t dg = m < n ? (uint32_t)(sortable(keys[e]) >> shift) & 255u : 256u;
                const uint32_t peers = __match_any_sync(0xffffffffu, dg);
                const uint32_t b0 = dg < 256u ? Hw[dg] : 0u;
                const uint32_t rank = b0 + __popc(peers & lt_mask);
                __syncwarp();
                if (dg < 256u && (peers & lt_mask) == 0) Hw[dg] = b0 + __popc(peers);
                __syncwarp();
                if (m < n) b[rank] = e;
            }
            __syncthreads();
        }
        int *t = a;
        a = b;
        b = t;
    }
    // 8 passes: the sorted order is back in the first array
}

template <bool NF, bool SCALE, bool DIGEST>
__global__ void __launch_bounds__(kTimeThreads, 2) time_kernel_large(
    const GeomParams g, const double *__restrict__ atoms, const double *__restrict__ times, int n, double c,
    double tau, double *__restrict__ out, WsHeader *__restrict__ hdr, int order_pixel, int *__restrict__ order_out,
    double *__restrict__ keys_out, unsigned char *__restrict__ slices, int n_slices, uint64_t *__restrict__ digest) {
    if ((int)blockIdx.x >= n_slices) return;  // one workspace slice per CTA
    extern __shared__ __align__(16) unsigned char smem[];
    uint32_t *cnt = reinterpret_cast<uint32_t *>(smem);
    uint32_t *H = cnt;                       // radix fallback: per-warp counters
    uint32_t *base = cnt + kTimeWarps * 256;  // and digit bases
    uint32_t *coarse = cnt + kLargeBuckets;
    __shared__ double scratch[128];
    __shared__ uint64_t s_dig[kTimeWarps];
    __shared__ int s_pix, s_flag;
    unsigned char *slice = slices + (size_t)blockIdx.x * large_slice_bytes(n);
    double *keys = reinterpret_cast<double *>(slice);
    SortRec *rec = reinterpret_cast<SortRec *>(slice + (size_t)n * 8);
    int *perm = reinterpret_cast<int *>(slice + (size_t)n * 24);
    int *perm2 = perm + n;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int npix = g.nx * g.ny;
    const int nb = large_buckets(n);
    const int per = (n + kTimeThreads - 1) / kTimeThreads;
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
        const double dn = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
        const double q0 = __ddiv_rn(dx, dn), q1 = __ddiv_rn(dy, dn), q2 = __dsub_rn(__ddiv_rn(dz, dn), 1.0);
        const double inv_tau = 1.0 / tau;
        double kmin = __longlong_as_double(0x7FF0000000000000ll), kmax = -kmin;
        for (int j = tid; j < n; j += kTimeThreads) {
            const double4 a = reinterpret_cast<const double4 *>(atoms)[j];
            double t, s, dist;
            arrival<NF, SCALE, false>(g, dx, dy, dz, dn, q0, q1, q2, a, times[j], c, 0.0, t, s, dist);
            kmin = fmin(kmin, t);
            kmax = fmax(kmax, t);
            keys[j] = t;
        }
        block_minmax(kmin, kmax, scratch + 96);
        __syncthreads();
        if (!bucket_sort_large(keys, rec, cnt, coarse, n, nb, kmin, kmax, scratch, &s_flag)) {
            radix_sort_large(keys, perm, perm2, n, H, base);
            for (int m = tid; m < n; m += kTimeThreads) rec[m] = SortRec{keys[perm[m]], perm[m], 0};
            __syncthreads();
        }
        if (p == order_pixel) {
            for (int m = tid; m < n; m += kTimeThreads) {
                order_out[m] = rec[m].idx;
                keys_out[m] = rec[m].key;
            }
        }
        const int m0 = tid * per;
        double Dm = 1.0, Br = 0.0, Bi = 0.0;
        double S1 = 0.0, S2r = 0.0, S2i = 0.0, S3 = 0.0;
        // neighbours' keys carried in registers, the next emitter row loaded one step ahead
        const double4 *atoms4 = reinterpret_cast<const double4 *>(atoms);
        double t_prev = m0 > 0 && m0 - 1 < n ? rec[m0 - 1].key : 0.0;
        SortRec r_next = SortRec{0.0, 0, 0};
        double4 a_next = make_double4(0.0, 0.0, 0.0, 0.0);
        if (m0 < n) {
            r_next = rec[m0];
            a_next = atoms4[r_next.idx];
        }
        uint64_t h = 0, pw = DIGEST && m0 < n ? digest_pow(m0) : 0;
        for (int i = 0; i < per; ++i) {
            const int m = m0 + i;
            if (m >= n) break;
            const double tj = r_next.key;
            const double4 a = a_next;
            if (DIGEST) {
                h += (uint64_t)(r_next.idx + 1) * pw;
                pw *= kDigestBase;
            }
            if (m + 1 < n) {
                r_next = rec[m + 1];
                if (i + 1 < per) a_next = atoms4[r_next.idx];
            }
            double s, dist, re, im;
            path_only<NF>(dx, dy, dz, dn, q0, q1, q2, a, s, dist);
            amplitude<NF, SCALE, false>(g.k, s, a.w, dist, re, im);
            const double dec = m == 0 ? 0.0 : exp(-__dsub_rn(tj, t_prev) * inv_tau);
            t_prev = tj;
            Dm *= dec;
            Br = fma(dec, Br, re);
            Bi = fma(dec, Bi, im);
            const double w = m < n - 1 ? (-tau / 2) * expm1(-2 * __dsub_rn(r_next.key, tj) * inv_tau) : tau / 2;
            const double wD = w * Dm;
            S1 = fma(wD, Dm, S1);
            S2r = fma(wD, Br, S2r);
            S2i = fma(wD, Bi, S2i);
            S3 = fma(w, fma(Br, Br, Bi * Bi), S3);
        }
        Affine incl = {Dm, Br, Bi};
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            Affine y;
            y.d = __shfl_up_sync(0xffffffffu, incl.d, o);
            y.br = __shfl_up_sync(0xffffffffu, incl.br, o);
            y.bi = __shfl_up_sync(0xffffffffu, incl.bi, o);
            if (lane >= o) incl = compose(y, incl);
        }
        __syncthreads();
        if (lane == 31) {
            scratch[warp * 3 + 0] = incl.d;
            scratch[warp * 3 + 1] = incl.br;
            scratch[warp * 3 + 2] = incl.bi;
        }
        __syncthreads();
        Affine wpre = {1.0, 0.0, 0.0};
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
        const double Xr = excl.br, Xi = excl.bi;
        double part = fma(fma(Xr, Xr, Xi * Xi), S1, fma(2.0, fma(Xr, S2r, Xi * S2i), S3));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            part += __shfl_down_sync(0xffffffffu, part, o);
            if (DIGEST) h += __shfl_down_sync(0xffffffffu, h, o);
        }
        __syncthreads();
        if (lane == 0) {
            scratch[64 + warp] = part;
            if (DIGEST) s_dig[warp] = h;
        }
        __syncthreads();
        if (tid == 0) {
            double tot = 0.0;
            uint64_t hh = 0;
            for (int w = 0; w < kTimeWarps; ++w) {
                tot += scratch[64 + w];
                if (DIGEST) hh += s_dig[w];
            }
            out[order_pixel >= 0 ? 0 : p] = tot;
            if (DIGEST && order_pixel < 0) digest[p] = hh;
        }
    }
}

template <bool NF, bool SCALE>
static void *time_kernel_large_ptr(bool digest) {
    return digest ? (void *)time_kernel_large<NF, SCALE, true> : (void *)time_kernel_large<NF, SCALE, false>;
}

template <bool NF, bool SCALE>
static void *time_kernel_ptr(bool digest) {
    return digest ? (void *)time_kernel<NF, SCALE, true> : (void *)time_kernel<NF, SCALE, false>;
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
    if (n > ((int64_t)1 << 28)) return set_error(IDIWF_ERR_UNSUPPORTED, "at most 2^28 emitters");
    if (!atoms || !times) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "atoms/times are NULL");
    if (reinterpret_cast<uintptr_t>(atoms) & 31) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "atoms must be 32-byte aligned");
    if (!(c > 0) || !(tau > 0)) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "c and tau must be positive");
    return IDIWF_OK;
}

static void *large_fn(const idiwf_geom *geom, bool digest = false) {
    const bool nf = geom->flags & IDIWF_NF, sc = geom->flags & IDIWF_SCALE;
    return nf ? (sc ? time_kernel_large_ptr<true, true>(digest) : time_kernel_large_ptr<true, false>(digest))
              : (sc ? time_kernel_large_ptr<false, true>(digest) : time_kernel_large_ptr<false, false>(digest));
}

// CTAs of the large-n kernel on this device, each owning one workspace
// slice.  The shared-memory attribute is set before the occupancy query, so
// the workspace size and the launch see the same count (both digest
// instances have the same resources).
static int large_ctas(const idiwf_geom *geom, int order_pixel) {
    if (order_pixel >= 0) return 1;
    void *fn = large_fn(geom);
    int dev = 0, sms = 148, occ = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLargeSmem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kTimeThreads, kLargeSmem) != cudaSuccess) {
        cudaGetLastError();
        occ = 1;
    }
    return std::max(1, std::min(geom->nx * geom->ny, sms * std::max(occ, 1)));
}

static size_t time_ws_bytes(const idiwf_geom *geom, int64_t n, int order_pixel) {
    if (n <= kTimeMaxN) return kWsDataOffset;
    return kWsDataOffset + (size_t)large_ctas(geom, order_pixel) * large_slice_bytes(n);
}

// digest: (nx, ny) uint64 order digests of every pixel, or NULL.
static idiwf_status time_launch(const idiwf_geom *geom, const double *atoms, const double *times, int64_t n,
                                double c, double tau, double *out, void *workspace, size_t workspace_bytes,
                                int order_pixel, int *order_out, double *keys_out, uint64_t *digest,
                                cudaStream_t stream) {
    const int slices_fit = n > kTimeMaxN ? large_ctas(geom, order_pixel) : 0;
    if (!workspace || workspace_bytes < time_ws_bytes(geom, n, order_pixel))
        return set_error(IDIWF_ERR_WORKSPACE, "workspace smaller than idiwf_time_workspace_size()");
    if (reinterpret_cast<uintptr_t>(workspace) & 255)
        return set_error(IDIWF_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    WsHeader *hdr = static_cast<WsHeader *>(workspace);
    const GeomParams g = make_geom(geom);
    const bool nf = geom->flags & IDIWF_NF, sc = geom->flags & IDIWF_SCALE;
    if (n > kTimeMaxN) {
        void *fl = large_fn(geom, digest != nullptr);
        IDIWF_CUDA_CHECK(cudaFuncSetAttribute(fl, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLargeSmem));
        IDIWF_CUDA_CHECK(cudaMemsetAsync(hdr, 0, 2 * sizeof(uint32_t), stream));
        // slices the workspace holds (the caller may pass more than the minimum)
        const size_t avail = (workspace_bytes - kWsDataOffset) / large_slice_bytes(n);
        int n_slices = (int)std::min<size_t>(avail, (size_t)1 << 20);
        const int grid = std::min(slices_fit, n_slices);
        n_slices = grid;
        int ni = (int)n;
        unsigned char *slices = static_cast<unsigned char *>(workspace) + kWsDataOffset;
        void *args[] = {(void *)&g, &atoms, &times, &ni, &c, &tau, &out, &hdr, &order_pixel, &order_out, &keys_out,
                        &slices, &n_slices, &digest};
        IDIWF_CUDA_CHECK(cudaLaunchKernel(fl, dim3(grid), dim3(kTimeThreads), args, kLargeSmem, stream));
        return IDIWF_OK;
    }
    const bool dg = digest != nullptr;
    void *fn = nf ? (sc ? time_kernel_ptr<true, true>(dg) : time_kernel_ptr<true, false>(dg))
                  : (sc ? time_kernel_ptr<false, true>(dg) : time_kernel_ptr<false, false>(dg));
    IDIWF_CUDA_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTimeSmem));
    // queue counter, error word, and the full-sort / given-up warm-start counts
    IDIWF_CUDA_CHECK(cudaMemsetAsync(hdr, 0, 5 * sizeof(uint32_t), stream));
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int npix = geom->nx * geom->ny;
    const int grid = order_pixel >= 0 ? 1 : std::min(npix, sms);
    // pixels per queue claim: an equal share of the detector per CTA, walked in
    // serpentine order (every pixel of a CTA but its first warm-starts from a
    // neighbour's order; the per-pixel cost hardly varies, so equal shares
    // balance)
    int chunk = (npix + grid - 1) / grid;
    int ni = (int)n;
    void *args[] = {(void *)&g, &atoms, &times, &ni, &c, &tau, &out, &hdr, &order_pixel, &order_out, &keys_out,
                    &digest, &chunk};
    IDIWF_CUDA_CHECK(cudaLaunchKernel(fn, dim3(grid), dim3(kTimeThreads), args, kTimeSmem, stream));
    return IDIWF_OK;
}

}  // namespace idiwf

using namespace idiwf;

extern "C" int64_t idiwf_time_max_emitters(void) { return kTimeMaxN; }

extern "C" size_t idiwf_time_workspace_size(const idiwf_geom *geom, int64_t n) {
    if (!geom || geom->nx <= 0 || geom->ny <= 0) return kWsDataOffset;
    return time_ws_bytes(geom, n, -1);
}

extern "C" idiwf_status idiwf_time_forward(const idiwf_geom *geom, const double *atoms, const double *times,
                                           int64_t n, double c, double tau, double *out, void *workspace,
                                           size_t workspace_bytes, cudaStream_t stream) {
    idiwf_status st = time_validate(geom, atoms, times, n, c, tau);
    if (st != IDIWF_OK) return st;
    if (!out) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "out is NULL");
    return time_launch(geom, atoms, times, n, c, tau, out, workspace, workspace_bytes, -1, nullptr, nullptr, nullptr,
                       stream);
}

extern "C" idiwf_status idiwf_time_forward_digest(const idiwf_geom *geom, const double *atoms, const double *times,
                                                  int64_t n, double c, double tau, double *out, uint64_t *digest,
                                                  void *workspace, size_t workspace_bytes, cudaStream_t stream) {
    idiwf_status st = time_validate(geom, atoms, times, n, c, tau);
    if (st != IDIWF_OK) return st;
    if (!out || !digest) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "out/digest is NULL");
    return time_launch(geom, atoms, times, n, c, tau, out, workspace, workspace_bytes, -1, nullptr, nullptr, digest,
                       stream);
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
    // the intensity of the pixel goes to a scratch slot of the workspace header
    double *scratch = reinterpret_cast<double *>(&static_cast<WsHeader *>(workspace)->pad[0]);
    return time_launch(geom, atoms, times, n, c, 1.0, scratch, workspace, workspace_bytes, ix * geom->ny + iy, order,
                       sorted_keys, nullptr, stream);
}
