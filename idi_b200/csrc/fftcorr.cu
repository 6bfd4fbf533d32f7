// FFT autocorrelation (idi/reconstruction/cusimple.py) by hand-written
// shared-memory FFTs, three passes per group of images: a tuned path for
// power-of-two shapes (fc_*), and a mixed-radix path for the reference's
// padded lengths fastlen(2 n) up to 4096 (fcg_*, with Bluestein's algorithm
// for the inverse of an odd last padded length and a 1D form for independent
// lines).  For larger shapes, the elementwise steps around cuFFT's transforms
// -- the power spectrum in place, the fftshift + centre crop fused with the
// normalisation -- and the correlator's running mean / variance.
#include <cmath>
#include <type_traits>

#include "idiwf_internal.cuh"

namespace idiwf {

template <typename T>
__global__ void power_kernel(T *__restrict__ z, int64_t n) {
    // one vector load and store per complex value
    using V = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
    V *zv = reinterpret_cast<V *>(z);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        V v = zv[i];
        v.x = v.x * v.x + v.y * v.y;
        v.y = T(0);
        zv[i] = v;
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

// The 2D case of crop_kernel without divisions: blockIdx.y is the output
// row (batch-major), threads run along the row.
template <typename T>
__global__ void crop2d_kernel(const T *__restrict__ full, int g0, int g1, int n0, int n1, const T *__restrict__ norm,
                              int mode, T threshold, T *__restrict__ out) {
    const int row = blockIdx.y;  // b * 2 n0 + i
    const int b = row / (2 * n0), i = row - b * 2 * n0;
    int j0 = (i - n0) % g0;
    if (j0 < 0) j0 += g0;
    const T *src = full + ((size_t)b * g0 + j0) * g1;
    T *dst = out + (size_t)row * 2 * n1;
    const T *nrm = norm ? norm + (size_t)i * 2 * n1 : nullptr;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < 2 * n1; c += gridDim.x * blockDim.x) {
        int j1 = (c - n1) % g1;
        if (j1 < 0) j1 += g1;
        T y = src[j1];
        if (nrm) {
            const T cn = nrm[c];
            if (mode == 0)
                y = cn < threshold ? T(NAN) : y / cn;
            else
                y = cn > threshold ? y / cn : T(0);
        }
        dst[c] = y;
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

// ---------------------------------------------------------------------------
// Hand-written FFT autocorrelation for power-of-two shapes: out =
// fftshift(irfft2(|rfft2(x, (2 n0, 2 n1))|^2)) -- the reference's padded
// length fastlen(2 n) is exactly 2 n for these shapes, so its centre crop is
// the whole shifted array -- optionally divided by a normalisation.  Three
// kernels per group of images, each made of shared-memory FFTs:
//   A  rows:    the real FFT of each input row (length G1 = 2 n1, zero-padded)
//               through a complex FFT of length H = n1 of (x[2k] + i x[2k+1])
//               and the split into even and odd parts; written transposed,
//               T[k][r] for k = 0..H (H + 1 columns of n0 rows);
//   B  columns: per column k, the complex FFT of length G0 = 2 n0 of T[k][.]
//               (rows n0.. are zero), the power |.|^2 and the inverse FFT (two
//               columns' real power spectra packed into one complex inverse),
//               written C[k][r] for rows r = 0..n0;
//   C  rows:    per row r = 0..n0, the inverse real FFT of the half spectrum
//               C[.][r] through a complex inverse FFT of length H, written with
//               the fftshift and the normalisation, twice: the autocorrelation
//               is point-symmetric, so row r also gives the mirrored row.
// The FFTs are Stockham auto-sort passes (Govindaraju et al., "High
// performance discrete Fourier transforms on graphics processors", SC 2008):
// natural order in and out, each pass a radix-16 (or 2/4/8 for the remainder)
// DFT of values held in registers, 16 per thread, with one shared-memory read
// and write per value per pass; slots are XOR-swizzled so that every pass's
// reads and writes are free of bank conflicts.  Inter-pass twiddles: one
// value exp(-2 pi i m / N) from a table (sincospi) per butterfly, its powers by
// multiplication in double precision.
// ---------------------------------------------------------------------------
template <typename T> struct Cx;
template <> struct Cx<double> { using t = double2; };
template <> struct Cx<float> { using t = float2; };

template <typename V> __device__ __forceinline__ V cx_mul(V a, V b) {
    V r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}
template <typename V> __device__ __forceinline__ V cx_add(V a, V b) {
    V r;
    r.x = a.x + b.x;
    r.y = a.y + b.y;
    return r;
}
template <typename V> __device__ __forceinline__ V cx_sub(V a, V b) {
    V r;
    r.x = a.x - b.x;
    r.y = a.y - b.y;
    return r;
}
template <typename V> __device__ __forceinline__ V cx_conj(V a) {
    a.y = -a.y;
    return a;
}
template <typename V> __device__ __forceinline__ V cx_zero() {
    V r;
    r.x = 0;
    r.y = 0;
    return r;
}

// Complex values per block of the FFT kernels (one 8192-point column takes
// 8192); values per thread E: 8 in FP64 (16 for the 8192-point column), 16
// in FP32 -- the block's values live in registers during a pass.
constexpr int kFcBlockElems = 4096;

// Shared-memory slot of complex value w.  A 128-byte bank row holds 8 (FP64)
// or 16 (FP32) values, and shared memory serves 8 (FP64) or 16 (FP32) threads
// of a warp at a time: one spare slot after every bank row of values makes
// the strided writes of every pass hit distinct banks within each such
// group, and rp spare slots per sequence (q = w >> logn) do the same for the
// row-interleaved loops that touch the same column of rpb rows at once.
struct FcSwz {
    int logn;  // sequence length (31: no sequence term)
    int rp;
};
template <typename V> __host__ __device__ constexpr int fc_lkc() { return sizeof(V) == 16 ? 3 : 4; }
template <typename V> __device__ __forceinline__ int fsw(int w, FcSwz z) {
    return w + (w >> fc_lkc<V>()) + (w >> z.logn) * z.rp;
}
// Layout of rpb interleaved rows of length 2^logn (rows shorter than a bank
// row get no row term).
template <typename V> __host__ __device__ inline FcSwz fc_rows_swz(int logn, int rpb) {
    const int kc = 1 << fc_lkc<V>();
    if (logn < fc_lkc<V>()) return FcSwz{31, 0};
    return FcSwz{logn, rpb < kc ? kc / rpb : 1};
}
// Shared-memory values for count sequences of 2^logn with layout z.
template <typename V> __host__ inline size_t fc_smem_values(int count, int logn, FcSwz z) {
    const size_t tot = (size_t)count << logn;
    return tot + (tot >> fc_lkc<V>()) + (z.logn == 31 ? 0 : (size_t)count * z.rp);
}

// d * exp(-/+ 2 pi i e / 16) for e = 0..7 (a constant after unrolling).
template <bool INV, typename V> __device__ __forceinline__ V mul_w16(V d, int e) {
    using T = decltype(d.x);
    constexpr double kC1 = 0.92387953251128675613;  // cos(pi / 8)
    constexpr double kS1 = 0.38268343236508977173;  // sin(pi / 8)
    constexpr double kH = 0.70710678118654752440;   // sqrt(1 / 2)
    double c, s;
    switch (e) {
        case 0: return d;
        case 4: {
            V r;
            r.x = INV ? -d.y : d.y;
            r.y = INV ? d.x : -d.x;
            return r;
        }
        case 1: c = kC1; s = kS1; break;
        case 2: c = kH; s = kH; break;
        case 3: c = kS1; s = kC1; break;
        case 5: c = -kS1; s = kC1; break;
        case 6: c = -kH; s = kH; break;
        default: c = -kC1; s = kS1; break;
    }
    const T tc = (T)c, ts = INV ? (T)s : (T)-s;
    V r;
    r.x = d.x * tc - d.y * ts;
    r.y = d.x * ts + d.y * tc;
    return r;
}

__host__ __device__ constexpr int brevc(int r, int R) {
    int o = 0;
    for (int b = 1; b < R; b <<= 1) o = (o << 1) | ((r & b) ? 1 : 0);
    return o;
}

// In-register R-point DFT (R = 2, 4, 8, 16): radix-2 decimation in frequency,
// X[q] ends in v[brevc(q, R)].
template <int R, bool INV, typename V> __device__ __forceinline__ void dft_reg(V *v) {
#pragma unroll
    for (int half = R / 2; half >= 1; half >>= 1) {
#pragma unroll
        for (int base = 0; base < R; base += 2 * half) {
#pragma unroll
            for (int j = 0; j < half; ++j) {
                const V a = v[base + j], b = v[base + j + half];
                v[base + j] = cx_add(a, b);
                v[base + j + half] = mul_w16<INV>(cx_sub(a, b), j * (16 / (2 * half)));
            }
        }
    }
}

// v[r] *= w^r, r = 1..R-1; the powers in double precision.
template <int R, typename V> __device__ __forceinline__ void twiddle_powers(V *v, double2 w) {
    using T = decltype(v[0].x);
    double2 p = w;
#pragma unroll
    for (int r = 1; r < R; ++r) {
        V q;
        q.x = (T)p.x;
        q.y = (T)p.y;
        v[r] = cx_mul(v[r], q);
        if (r + 1 < R) p = cx_mul(p, w);
    }
}

// First passes from global memory take one butterfly at a time in FP64,
// where registers bound the blocks per SM; FP32 keeps all its loads in
// flight.
template <typename T> constexpr bool kFcOneAtATime = sizeof(T) == 8;

// Loader of a pass that reads shared memory (never called).
template <typename V> struct FcNoLoad {
    __device__ V operator()(int, int) const { return cx_zero<V>(); }
};

// One Stockham pass over `count` sequences of length n = 2^logn at S: each
// butterfly g (thread t takes g = t, t + blockDim, ...) reads
// in[j + r n/R] (from shared memory, or from `ld(sequence, index)` for a first
// pass), multiplies by exp(-/+ 2 pi i (j mod Ns) r / (Ns R)), takes the R-point
// DFT and writes out[(j - j mod Ns) R + j mod Ns + q Ns].  In place: all reads
// of the block come before its writes, except for a first pass whose loader
// reads global memory only (LD_GLOBAL), which takes one butterfly at a time.
template <typename V, int R, int E, bool INV, bool LOADER, bool LD_GLOBAL, class Ld>
__device__ __forceinline__ void fc_pass(V *S, FcSwz z, int logn, int count, int Ns, const double2 *__restrict__ tw,
                                        int N, const Ld &ld) {
    constexpr int NB = E / R;
    constexpr int LR = R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : 4;
    const int n = 1 << logn, lognb = logn - LR, nb = 1 << lognb, total = count << lognb;
    if constexpr (LOADER && LD_GLOBAL) {
        // Ns = 1: no twiddles
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int g = threadIdx.x + b * blockDim.x;
            if (g < total) {
                const int q = g >> lognb, j = g & (nb - 1);
                V v[R];
#pragma unroll
                for (int r = 0; r < R; ++r) v[r] = ld(q, j + r * nb);
                dft_reg<R, INV>(v);
                const int base = q * n + j * R;
#pragma unroll
                for (int r = 0; r < R; ++r) S[fsw<V>(base + r, z)] = v[brevc(r, R)];
            }
        }
        __syncthreads();
    } else {
        V v[E];
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int g = threadIdx.x + b * blockDim.x;
            if (g < total) {
                const int q = g >> lognb, j = g & (nb - 1);
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if constexpr (LOADER)
                        v[b * R + r] = ld(q, j + r * nb);
                    else
                        v[b * R + r] = S[fsw<V>(q * n + j + r * nb, z)];
                }
            }
        }
        __syncthreads();
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int g = threadIdx.x + b * blockDim.x;
            if (g < total) {
                const int q = g >> lognb, j = g & (nb - 1), k = j & (Ns - 1);
                if (Ns > 1) {
                    double2 w = __ldg(&tw[k * (N / (Ns * R))]);
                    if (INV) w.y = -w.y;
                    twiddle_powers<R>(&v[b * R], w);
                }
                dft_reg<R, INV>(&v[b * R]);
                const int base = q * n + (j - k) * R + k;
#pragma unroll
                for (int r = 0; r < R; ++r) S[fsw<V>(base + r * Ns, z)] = v[b * R + brevc(r, R)];
            }
        }
        __syncthreads();
    }
}

// The FFT of `count` sequences of length 2^logn in place at S (natural order
// in and out), E values per thread (count << logn <= E * blockDim.x); the
// first pass reads through `ld` when from_loader.
template <typename V, int E, bool INV, bool LD_GLOBAL, class Ld>
__device__ __forceinline__ void fc_fft(V *S, FcSwz z, int logn, int count, const double2 *__restrict__ tw, int N,
                                       const Ld &ld, bool from_loader) {
    constexpr int LMAX = E >= 16 ? 4 : 3;
    int Ns = 1;
    bool first = from_loader;
    const int rem = logn % LMAX;
#define FC_RUN(RR)                                                                          \
    do {                                                                                    \
        if (first)                                                                          \
            fc_pass<V, RR, E, INV, true, LD_GLOBAL>(S, z, logn, count, Ns, tw, N, ld);      \
        else                                                                                \
            fc_pass<V, RR, E, INV, false, false>(S, z, logn, count, Ns, tw, N, ld);         \
        first = false;                                                                      \
        Ns *= RR;                                                                           \
    } while (0)
    if (rem == 1) FC_RUN(2);
    else if (rem == 2) FC_RUN(4);
    else if (rem == 3) { if constexpr (LMAX == 4) FC_RUN(8); }
    for (int p = 0; p < logn / LMAX; ++p) FC_RUN(1 << LMAX);
#undef FC_RUN
}

// Pass A: rpb rows per block, one image per blockIdx.y.  x: n0 x n1 real per
// image; T: (H+1) x n0 complex per image (t_img values apart).
template <typename T, int E>
__global__ void __launch_bounds__(512, (sizeof(T) == 8 && E == 8) ? 2 : 1) fc_rows_fwd(const T *__restrict__ x, int n0, int n1, int logh, int rpb,
                                                   const double2 *__restrict__ tw, int N,
                                                   typename Cx<T>::t *__restrict__ Tt, size_t t_img) {
    using V = typename Cx<T>::t;
    extern __shared__ __align__(16) unsigned char fsm[];
    V *S = reinterpret_cast<V *>(fsm);
    const int H = 1 << logh, r0 = blockIdx.x * rpb;
    x += (size_t)blockIdx.y * n0 * n1;
    Tt += (size_t)blockIdx.y * t_img;
    // (x[2k], x[2k+1]) in one load: n1 is even and x is aligned to two values;
    // k >= H/2 is the zero padding
    auto ld = [&](int q, int k) -> V {
        V z = cx_zero<V>();
        const int r = r0 + q;
        if (r < n0 && k < (H >> 1)) z = reinterpret_cast<const V *>(x + (size_t)r * n1)[k];
        return z;
    };
    const FcSwz z = fc_rows_swz<V>(logh, rpb);
    fc_fft<V, E, false, kFcOneAtATime<T>>(S, z, logh, rpb, tw, N, ld, true);
    // X[k] = (Z[k] + conj Z[H-k]) / 2 + W^k (Z[k] - conj Z[H-k]) / (2i), W = exp(-2 pi i / G1)
    const int wstep = N / (2 * H), lrpb = 31 - __clz(rpb);
    for (int idx = threadIdx.x; idx < (H + 1) * rpb; idx += blockDim.x) {
        const int k = idx >> lrpb, rr = idx & (rpb - 1), r = r0 + rr;
        if (r >= n0) continue;
        const V zk = S[fsw<V>(rr * H + (k & (H - 1)), z)], zc = cx_conj(S[fsw<V>(rr * H + ((H - k) & (H - 1)), z)]);
        const V e = cx_add(zk, zc), d = cx_sub(zk, zc);
        V o;  // d / (2i) = (d.y, -d.x) / 2
        o.x = d.y;
        o.y = -d.x;
        const double2 wd = __ldg(&tw[k * wstep]);
        V w;
        w.x = (T)wd.x;
        w.y = (T)wd.y;
        const V wo = cx_mul(w, o);
        V X;
        X.x = T(0.5) * (e.x + wo.x);
        X.y = T(0.5) * (e.y + wo.y);
        Tt[(size_t)k * n0 + r] = X;
    }
}

// Pass B: cpb columns per block (cpb = 1 for 8192-point columns), one image
// per blockIdx.y.  The forward FFTs of the cpb columns (first pass straight
// from T), then one inverse FFT per pair of columns of the packed power
// spectra Z = P_k + i P_k+1 (both real; P_k+1 = 0 without a partner),
// unpacked by Hermitian symmetry:
// IFFT(P_k)[r] = (z[r] + conj z[-r]) / 2, IFFT(P_k+1)[r] = (z[r] - conj z[-r]) / (2i);
// rows 0..n0 only (the rest follows from the point symmetry in pass C).
// The inverse runs on the first npair * G0 / E threads.
template <typename T, int E>
__global__ void __launch_bounds__(512, (sizeof(T) == 8 && E == 8) ? 2 : 1) fc_cols(const typename Cx<T>::t *__restrict__ Tt, size_t t_img, int n0,
                                               int ncols, int logg0, int cpb, const double2 *__restrict__ tw, int N,
                                               typename Cx<T>::t *__restrict__ C, size_t c_img) {
    using V = typename Cx<T>::t;
    extern __shared__ __align__(16) unsigned char fsm[];
    V *S = reinterpret_cast<V *>(fsm);
    const int G0 = 1 << logg0, k0 = blockIdx.x * cpb;
    Tt += (size_t)blockIdx.y * t_img;
    C += (size_t)blockIdx.y * c_img;
    auto ldT = [&](int q, int r) -> V {
        V z = cx_zero<V>();
        const int col = k0 + q;
        if (r < n0 && col < ncols) z = Tt[(size_t)col * n0 + r];
        return z;
    };
    const FcSwz sz{31, 0};
    fc_fft<V, E, false, kFcOneAtATime<T>>(S, sz, logg0, cpb, tw, N, ldT, true);
    const int npair = (cpb + 1) >> 1;
    auto ldP = [&](int q, int r) -> V {
        const V u = S[fsw<V>(2 * q * G0 + r, sz)];
        V z;
        z.x = u.x * u.x + u.y * u.y;
        z.y = T(0);
        if (2 * q + 1 < cpb) {
            const V w = S[fsw<V>((2 * q + 1) * G0 + r, sz)];
            z.y = w.x * w.x + w.y * w.y;
        }
        return z;
    };
    fc_fft<V, E, true, false>(S, sz, logg0, npair, tw, N, ldP, true);
    const T half = T(0.5) / (T)G0;
    int q = threadIdx.x / (n0 + 1), r = threadIdx.x - q * (n0 + 1);
    for (; q < npair; r += blockDim.x, q += r / (n0 + 1), r %= (n0 + 1)) {
        const V zp = S[fsw<V>(q * G0 + r, sz)], zm = cx_conj(S[fsw<V>(q * G0 + ((G0 - r) & (G0 - 1)), sz)]);
        const int col = k0 + 2 * q;
        if (col < ncols) {
            V c0;
            c0.x = (zp.x + zm.x) * half;
            c0.y = (zp.y + zm.y) * half;
            C[(size_t)col * (n0 + 1) + r] = c0;
        }
        if (2 * q + 1 < cpb && col + 1 < ncols) {
            V c1;  // (zp - zm) / (2i) = ((zp - zm).y, -(zp - zm).x) / 2
            c1.x = (zp.y - zm.y) * half;
            c1.y = -(zp.x - zm.x) * half;
            C[(size_t)(col + 1) * (n0 + 1) + r] = c1;
        }
    }
}

// Pass C: rpb rows per block of rows 0..n0, one image per blockIdx.y; the
// inverse real FFT of each row's half spectrum, then the fftshift (row r to
// (r + n0) mod G0, column c to (c + n1) mod G1) and, by the point symmetry of
// an autocorrelation (A[-d] = A[d]), the mirrored row n0 - r with column c at
// (n1 - c) mod G1; each thread stores two adjacent columns at once.  The
// normalisation at each output position: mode 0 divides by norm (NaN below
// threshold), mode 1 divides by norm (0 at or below threshold), mode 2 by the
// pair count (n0 - |i - n0|)(n1 - |j - n1|) (NaN below threshold), mode -1
// none.
template <typename T, int E>
__global__ void __launch_bounds__(512, (sizeof(T) == 8 && E == 8) ? 2 : 1) fc_rows_inv(const typename Cx<T>::t *__restrict__ C, size_t c_img, int n0,
                                                   int n1, int logh, int rpb, const double2 *__restrict__ tw, int N,
                                                   const T *__restrict__ norm, int mode, T threshold,
                                                   T *__restrict__ out) {
    using V = typename Cx<T>::t;
    extern __shared__ __align__(16) unsigned char fsm[];
    V *S = reinterpret_cast<V *>(fsm);
    const int H = 1 << logh, G1 = 2 * H, G0 = 2 * n0, r0 = blockIdx.x * rpb;
    C += (size_t)blockIdx.y * c_img;
    out += (size_t)blockIdx.y * G0 * G1;
    const int wstep = N / G1;
    const FcSwz sz = fc_rows_swz<V>(logh, rpb);
    // Z[k] = (Y[k] + conj Y[H-k]) + i W^-k (Y[k] - conj Y[H-k]); rows fastest,
    // the rpb rows of one k are contiguous in C
    const int lrpb = 31 - __clz(rpb);
    for (int idx = threadIdx.x; idx < rpb * H; idx += blockDim.x) {
        const int k = idx >> lrpb, rr = idx & (rpb - 1), r = r0 + rr;
        V z = cx_zero<V>();
        if (r <= n0) {
            const V yk = C[(size_t)k * (n0 + 1) + r], yc = cx_conj(C[(size_t)(H - k) * (n0 + 1) + r]);
            const V e = cx_add(yk, yc), d = cx_sub(yk, yc);
            const double2 wdd = __ldg(&tw[k * wstep]);
            V w;
            w.x = (T)wdd.x;
            w.y = (T)-wdd.y;
            const V wd = cx_mul(w, d);
            z.x = e.x - wd.y;
            z.y = e.y + wd.x;
        }
        S[fsw<V>(rr * H + k, sz)] = z;
    }
    __syncthreads();
    fc_fft<V, E, true, false>(S, sz, logh, rpb, tw, N, FcNoLoad<V>{}, false);
    const T scale = T(1) / (T)G1;  // the inverse's 1/H and the split's 1/2
    auto fix = [&](int i, int j, T y) -> T {
        if (mode == 0 || mode == 1) {
            const T cn = norm[(size_t)i * G1 + j];
            return mode == 0 ? (cn < threshold ? T(NAN) : y / cn) : (cn > threshold ? y / cn : T(0));
        }
        if (mode == 2) {
            const T cn = (T)((int64_t)(n0 - abs(i - n0)) * (n1 - abs(j - n1)));
            return cn < threshold ? T(NAN) : y / cn;
        }
        return y;
    };
    auto put2 = [&](int i, int j, T y0, T y1) {  // columns j (even), j + 1
        V p;
        p.x = fix(i, j, y0);
        p.y = fix(i, j + 1, y1);
        *reinterpret_cast<V *>(out + (size_t)i * G1 + j) = p;
    };
    for (int idx = threadIdx.x; idx < rpb * H; idx += blockDim.x) {
        const int rr = idx >> logh, k = idx & (H - 1), r = r0 + rr;
        if (r > n0) continue;
        // value k holds columns c = 2k (x) and 2k + 1 (y)
        const V z = S[fsw<V>(rr * H + k, sz)];
        const int i = (r + n0) & (G0 - 1), im = (n0 - r) & (G0 - 1);
        put2(i, (2 * k + n1) & (G1 - 1), z.x * scale, z.y * scale);
        if (im != i) {
            // mirrored columns (n1 - 2k, n1 - 2k + 1) hold c = 2k and c = 2k - 1
            const V zp = S[fsw<V>(rr * H + ((k - 1) & (H - 1)), sz)];
            put2(im, (n1 - 2 * k) & (G1 - 1), z.x * scale, zp.y * scale);
        }
    }
}

// tw[m] = exp(-2 pi i m / N), m = 0..N-1, in double precision for both dtypes
__global__ void fc_twiddle_kernel(double2 *tw, int N) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= N) return;
    double sn, cs;
    sincospi(-2.0 * (double)m / (double)N, &sn, &cs);
    tw[m] = make_double2(cs, sn);
}

// ---------------------------------------------------------------------------
// General lengths: the reference pads each axis to fastlen(2 n) (factors 2,
// 3, 5, 7, 11).  The same three kernels, with mixed-radix Stockham passes
// (radix 8/4/2 and 3, 5, 7, 11), rows packed in pairs as x_a + i x_b for the
// row FFT, and the inverse along rows of length L1 = G1 through a complex
// inverse of L1/2 values (the real parts only at frequencies 0 and L1/2, as
// a c2r transform).  The output is the centre crop (i - n0) mod G0,
// (j - n1) mod L1 of the shifted array.  An odd G1 is not taken: the
// reference's inverse then has length G1 - 1, which is never a product of 2,
// 3, 5, 7, 11 (it would be a smaller padded length).
// ---------------------------------------------------------------------------
// {cos, sin}(2 pi m / R) for R = 3, 5, 7, 11, m = 0..R-1 (offsets 0, 3, 8, 15)
__constant__ double2 kFcgOdd[26] = {
    {1.0, 0.0},
    {-5.0e-1, 8.66025403784438646764e-1},
    {-5.0e-1, -8.66025403784438646764e-1},
    {1.0, 0.0},
    {3.09016994374947424102e-1, 9.51056516295153572116e-1},
    {-8.09016994374947424102e-1, 5.87785252292473129169e-1},
    {-8.09016994374947424102e-1, -5.87785252292473129169e-1},
    {3.09016994374947424102e-1, -9.51056516295153572116e-1},
    {1.0, 0.0},
    {6.23489801858733530525e-1, 7.81831482468029808708e-1},
    {-2.22520933956314404289e-1, 9.74927912181823607018e-1},
    {-9.00968867902419126236e-1, 4.33883739117558120476e-1},
    {-9.00968867902419126236e-1, -4.33883739117558120476e-1},
    {-2.22520933956314404289e-1, -9.74927912181823607018e-1},
    {6.23489801858733530525e-1, -7.81831482468029808708e-1},
    {1.0, 0.0},
    {8.41253532831181168862e-1, 5.40640817455597582108e-1},
    {4.15415013001886425529e-1, 9.09631995354518371412e-1},
    {-1.42314838273285140444e-1, 9.89821441880932732376e-1},
    {-6.54860733945285064057e-1, 7.55749574354258283774e-1},
    {-9.5949297361449738989e-1, 2.81732556841429697711e-1},
    {-9.5949297361449738989e-1, -2.81732556841429697711e-1},
    {-6.54860733945285064057e-1, -7.55749574354258283774e-1},
    {-1.42314838273285140444e-1, -9.89821441880932732376e-1},
    {4.15415013001886425529e-1, -9.09631995354518371412e-1},
    {8.41253532831181168862e-1, -5.40640817455597582108e-1},
};
template <int R> __host__ __device__ constexpr int fcg_odd_off() { return R == 3 ? 0 : R == 5 ? 3 : R == 7 ? 8 : 15; }

// Register holding output q of fcg_dft<R>: bit-reversed for R = 2^m.
template <int R> __host__ __device__ constexpr int fcg_out(int q) { return (R & (R - 1)) == 0 ? brevc(q, R) : q; }

// R-point DFT in registers, output q in v[fcg_out<R>(q)]; odd R by the
// symmetric pairs x_k +- x_{R-k} (real and imaginary halves), R = 2^m by
// dft_reg.
template <int R, bool INV, typename V> __device__ __forceinline__ void fcg_dft(V *v) {
    using T = decltype(v[0].x);
    if constexpr ((R & (R - 1)) == 0) {
        dft_reg<R, INV>(v);
    } else {
        constexpr int h = (R - 1) / 2, off = fcg_odd_off<R>();
        V a[h], b[h];
        V x0 = v[0], X0 = v[0];
#pragma unroll
        for (int k = 1; k <= h; ++k) {
            a[k - 1] = cx_add(v[k], v[R - k]);
            b[k - 1] = cx_sub(v[k], v[R - k]);
            X0 = cx_add(X0, a[k - 1]);
        }
        v[0] = X0;
#pragma unroll
        for (int q = 1; q <= h; ++q) {
            V re = x0, im = cx_zero<V>();
#pragma unroll
            for (int k = 1; k <= h; ++k) {
                const double2 cs = kFcgOdd[off + (k * q) % R];
                re.x += a[k - 1].x * (T)cs.x;
                re.y += a[k - 1].y * (T)cs.x;
                im.x += b[k - 1].x * (T)cs.y;
                im.y += b[k - 1].y * (T)cs.y;
            }
            // sum_k x_k W^{kq} = re -/+ i im (W = exp(-/+ 2 pi i / R))
            V mi;  // -i * im
            mi.x = im.y;
            mi.y = -im.x;
            v[q] = INV ? cx_sub(re, mi) : cx_add(re, mi);
            v[R - q] = INV ? cx_add(re, mi) : cx_sub(re, mi);
        }
    }
}

// Radices of one general length n (pass order: 11, 7, 5, 3, then 8s, then
// the remaining 4 or 2).
constexpr int kFcgMaxPasses = 14;
struct FcgRad {
    int n, np;
    int r[kFcgMaxPasses];
};

// Slot of value i of sequence q: sequences `stride` slots apart, one spare
// slot per 8 (FP64) or 16 (FP32) values.
template <typename V> __device__ __forceinline__ int fcg_slot(int q, int i, int stride) {
    return q * stride + i + (i >> fc_lkc<V>());
}

// (a, b) = divmod(i, nb) for i = start, start + step, ...: one division at
// the start, then additions.
struct FcgIdx {
    int a, b, da, db, nb;
    __device__ __forceinline__ FcgIdx(int start, int step, int nb_) : nb(nb_) {
        a = start / nb;
        b = start - a * nb;
        da = step / nb;
        db = step - da * nb;
    }
    __device__ __forceinline__ void next() {
        a += da;
        b += db;
        if (b >= nb) {
            b -= nb;
            ++a;
        }
    }
};

// Out-of-place Stockham pass of radix R (in -> out), one butterfly of R
// values in registers per loop iteration.
template <typename V, int R, bool INV>
__device__ __forceinline__ void fcg_pass(const V *in, V *out, int stride, int n, int count, int Ns,
                                         const double2 *__restrict__ tab, int ntab) {
    const int nb = n / R, total = count * nb, tstep = ntab / (Ns * R);
    FcgIdx it(threadIdx.x, blockDim.x, nb);
    // k = j mod Ns (nb is a multiple of Ns, so the wrap of j keeps k)
    const int dk = it.db % Ns;
    int k = it.b % Ns;
    for (int g = threadIdx.x; g < total; g += blockDim.x, it.next(), k = (k + dk >= Ns) ? k + dk - Ns : k + dk) {
        const int q = it.a, j = it.b;
        V v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = in[fcg_slot<V>(q, j + r * nb, stride)];
        if (Ns > 1) {
            double2 w = __ldg(&tab[k * tstep]);
            if (INV) w.y = -w.y;
            twiddle_powers<R>(v, w);
        }
        fcg_dft<R, INV>(v);
        const int base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) out[fcg_slot<V>(q, base + r * Ns, stride)] = v[fcg_out<R>(r)];
    }
}

// The FFT of `count` sequences of length rad.n: the values from `ld` (or
// already in A) go through the passes between buffers A and B; returns the
// buffer holding the result.
template <typename V, bool INV, class Ld>
__device__ __forceinline__ V *fcg_fft(V *A, V *B, int stride, const FcgRad &rad, int count,
                                      const double2 *__restrict__ tab, int ntab, const Ld &ld, bool from_loader) {
    const int n = rad.n;
    if (from_loader) {
        FcgIdx it(threadIdx.x, blockDim.x, n);
        for (int idx = threadIdx.x; idx < count * n; idx += blockDim.x, it.next())
            A[fcg_slot<V>(it.a, it.b, stride)] = ld(it.a, it.b);
        __syncthreads();
    }
    V *in = A, *out = B;
    int Ns = 1;
    for (int p = 0; p < rad.np; ++p) {
        const int R = rad.r[p];
        switch (R) {
            case 2: fcg_pass<V, 2, INV>(in, out, stride, n, count, Ns, tab, ntab); break;
            case 3: fcg_pass<V, 3, INV>(in, out, stride, n, count, Ns, tab, ntab); break;
            case 4: fcg_pass<V, 4, INV>(in, out, stride, n, count, Ns, tab, ntab); break;
            case 5: fcg_pass<V, 5, INV>(in, out, stride, n, count, Ns, tab, ntab); break;
            case 7: fcg_pass<V, 7, INV>(in, out, stride, n, count, Ns, tab, ntab); break;
            case 8: fcg_pass<V, 8, INV>(in, out, stride, n, count, Ns, tab, ntab); break;
            default: fcg_pass<V, 11, INV>(in, out, stride, n, count, Ns, tab, ntab); break;
        }
        __syncthreads();
        V *t = in;
        in = out;
        out = t;
        Ns *= R;
    }
    return in;
}

// Bluestein's algorithm for the inverse along rows when L1/2 has a prime
// factor above 11 (an odd G1, L1 = G1 - 1): with c_m = exp(pi i m^2 / N),
//     sum_n Z_n exp(2 pi i k n / N) = c_k sum_n (Z_n c_n) conj(c_{k-n}),
// a cyclic convolution of length M = fastlen(2N - 1) done with the FFTs
// above; the filter's spectrum Bf = FFT(conj c, wrapped) / M is made once
// per call.
__global__ void fcg_chirp_kernel(double2 *c, int N) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= N) return;
    const int64_t e = ((int64_t)m * m) % (2 * (int64_t)N);  // exact: the angle pi e / N
    double sn, cs;
    sincospi((double)e / (double)N, &sn, &cs);
    c[m] = make_double2(cs, sn);
}

__global__ void __launch_bounds__(512) fcg_blue_filter_kernel(const double2 *__restrict__ c, int N, FcgRad radM,
                                                              int stride, const double2 *__restrict__ twM,
                                                              double2 *__restrict__ Bf) {
    extern __shared__ __align__(16) unsigned char fsm[];
    double2 *S = reinterpret_cast<double2 *>(fsm);
    const int M = radM.n;
    auto ld = [&](int, int i) -> double2 {
        const int m = i < N ? i : (M - i < N ? M - i : -1);
        if (m < 0) return make_double2(0.0, 0.0);
        return make_double2(c[m].x, -c[m].y);
    };
    const double2 *F = fcg_fft<double2, false>(S, S + stride, stride, radM, 1, twM, M, ld, true);
    const double inv = 1.0 / (double)M;
    for (int i = threadIdx.x; i < M; i += blockDim.x) {
        const double2 v = F[fcg_slot<double2>(0, i, stride)];
        Bf[i] = make_double2(v.x * inv, v.y * inv);
    }
}

// Launch bounds of the general kernels: FP64 blocks (2048 values) fit two
// per SM and take 256 threads -- the bound of 512 leaves them 128 registers;
// FP32 blocks (4096 values) take at most 256 threads and are held to 85
// registers for three blocks per SM (measured 16-20 % faster than two).
template <typename T> constexpr int kFcgMaxThreads = sizeof(T) == 8 ? 512 : 256;
template <typename T> constexpr int kFcgMinBlocks = sizeof(T) == 8 ? 1 : 3;

// Pass A (general): ppb pairs of rows per block, one image per blockIdx.y;
// rows 2p, 2p+1 as one complex sequence of length G1 (zero-padded from n1),
// split by Hermitian symmetry into the two real spectra, columns k = 0..m-1
// (m = G1/2 + 1) written to T[k][r].
template <typename T>
__global__ void __launch_bounds__(kFcgMaxThreads<T>, kFcgMinBlocks<T>) fcg_rows_fwd(const T *__restrict__ x, int n0, int n1, int ppb, FcgRad rad,
                                                    int stride, const double2 *__restrict__ twg1, int m,
                                                    typename Cx<T>::t *__restrict__ Tt, size_t t_img) {
    using V = typename Cx<T>::t;
    extern __shared__ __align__(16) unsigned char fsm[];
    V *S = reinterpret_cast<V *>(fsm);
    const int G1 = rad.n, p0 = blockIdx.x * ppb;
    x += (size_t)blockIdx.y * n0 * n1;
    Tt += (size_t)blockIdx.y * t_img;
    auto ld = [&](int q, int c) -> V {
        V z = cx_zero<V>();
        const int ra = 2 * (p0 + q);
        if (c < n1) {
            if (ra < n0) z.x = x[(size_t)ra * n1 + c];
            if (ra + 1 < n0) z.y = x[(size_t)(ra + 1) * n1 + c];
        }
        return z;
    };
    const V *Z = fcg_fft<V, false>(S, S + ppb * stride, stride, rad, ppb, twg1, G1, ld, true);
    // X_a[k] = (Z[k] + conj Z[-k]) / 2, X_b[k] = (Z[k] - conj Z[-k]) / (2i); pairs fastest
    FcgIdx it(threadIdx.x, blockDim.x, ppb);
    for (int idx = threadIdx.x; idx < m * ppb; idx += blockDim.x, it.next()) {
        const int k = it.a, q = it.b, ra = 2 * (p0 + q);
        if (ra >= n0) continue;
        const V zk = Z[fcg_slot<V>(q, k, stride)];
        const V zc = cx_conj(Z[fcg_slot<V>(q, k == 0 ? 0 : G1 - k, stride)]);
        V xa;
        xa.x = T(0.5) * (zk.x + zc.x);
        xa.y = T(0.5) * (zk.y + zc.y);
        Tt[(size_t)k * n0 + ra] = xa;
        if (ra + 1 < n0) {
            V xb;
            xb.x = T(0.5) * (zk.y - zc.y);
            xb.y = -T(0.5) * (zk.x - zc.x);
            Tt[(size_t)k * n0 + ra + 1] = xb;
        }
    }
}

// Pass B (general): as fc_cols for a column length G0 = rad.n of any
// factorisation.
template <typename T>
__global__ void __launch_bounds__(kFcgMaxThreads<T>, kFcgMinBlocks<T>) fcg_cols(const typename Cx<T>::t *__restrict__ Tt, size_t t_img, int n0,
                                                int ncols, int cpb, FcgRad rad, int stride,
                                                const double2 *__restrict__ twg0, typename Cx<T>::t *__restrict__ C,
                                                size_t c_img) {
    using V = typename Cx<T>::t;
    extern __shared__ __align__(16) unsigned char fsm[];
    V *S = reinterpret_cast<V *>(fsm);
    const int G0 = rad.n, k0 = blockIdx.x * cpb;
    Tt += (size_t)blockIdx.y * t_img;
    C += (size_t)blockIdx.y * c_img;
    auto ldT = [&](int q, int r) -> V {
        V z = cx_zero<V>();
        const int col = k0 + q;
        if (r < n0 && col < ncols) z = Tt[(size_t)col * n0 + r];
        return z;
    };
    V *S2 = S + cpb * stride;
    V *F = fcg_fft<V, false>(S, S2, stride, rad, cpb, twg0, G0, ldT, true);
    const int npair = (cpb + 1) >> 1;
    auto ldP = [&](int q, int r) -> V {
        const V u = F[fcg_slot<V>(2 * q, r, stride)];
        V z;
        z.x = u.x * u.x + u.y * u.y;
        z.y = T(0);
        if (2 * q + 1 < cpb) {
            const V w = F[fcg_slot<V>(2 * q + 1, r, stride)];
            z.y = w.x * w.x + w.y * w.y;
        }
        return z;
    };
    // the packed spectra load into the other buffer, then the passes run
    // between it and F
    const V *P = fcg_fft<V, true>(F == S ? S2 : S, F, stride, rad, npair, twg0, G0, ldP, true);
    const T half = T(0.5) / (T)G0;
    FcgIdx it(threadIdx.x, blockDim.x, n0 + 1);
    for (int idx = threadIdx.x; idx < npair * (n0 + 1); idx += blockDim.x, it.next()) {
        const int q = it.a, r = it.b;
        const V zp = P[fcg_slot<V>(q, r, stride)];
        const V zm = cx_conj(P[fcg_slot<V>(q, r == 0 ? 0 : G0 - r, stride)]);
        const int col = k0 + 2 * q;
        if (col < ncols) {
            V c0;
            c0.x = (zp.x + zm.x) * half;
            c0.y = (zp.y + zm.y) * half;
            C[(size_t)col * (n0 + 1) + r] = c0;
        }
        if (2 * q + 1 < cpb && col + 1 < ncols) {
            V c1;
            c1.x = (zp.y - zm.y) * half;
            c1.y = -(zp.x - zm.x) * half;
            C[(size_t)(col + 1) * (n0 + 1) + r] = c1;
        }
    }
}

// Pass C (general): rpb rows per block of rows 0..n0; the inverse real FFT
// of length L1 = 2 Hp through a complex inverse FFT of Hp values (the real
// parts only at frequencies 0 and L1/2, as a c2r transform), then the
// centre crop: output (i, j) of row r is column (j - n1) mod L1 for
// i = n0 + r (r < n0), and by point symmetry column (n1 - j) mod L1 for the
// mirrored row i = n0 - r.  Normalisation modes as fc_rows_inv.
// ONED: the autocorrelation of each of n0 lines on its own -- the half
// spectrum is the line's power |T[k][r]|^2 (C is pass A's T), and line r's
// result is output row r (pair count n1 - |j - n1|, norm of 2 n1 values).
// BLUE: the inverse of Hp values by Bluestein's algorithm through FFTs of
// length rad.n = M (chirp c, filter spectrum Bf); otherwise rad.n = Hp.
template <typename T, bool ONED, bool BLUE>
__global__ void __launch_bounds__(kFcgMaxThreads<T>, kFcgMinBlocks<T>) fcg_rows_inv(const typename Cx<T>::t *__restrict__ C, size_t c_img, int n0,
                                                    int n1, int Hp, int rpb, FcgRad rad, int stride,
                                                    const double2 *__restrict__ twl1, const double2 *__restrict__ twm,
                                                    const double2 *__restrict__ chirp,
                                                    const double2 *__restrict__ Bf, const T *__restrict__ norm,
                                                    int mode, T threshold, T *__restrict__ out) {
    using V = typename Cx<T>::t;
    extern __shared__ __align__(16) unsigned char fsm[];
    V *S = reinterpret_cast<V *>(fsm);
    V *S2 = S + rpb * stride;
    const int L1 = 2 * Hp, r0 = blockIdx.x * rpb, W = 2 * n1, NF = rad.n;
    const int rows = ONED ? n0 : n0 + 1, cst = ONED ? n0 : n0 + 1;
    C += (size_t)blockIdx.y * c_img;
    out += (size_t)blockIdx.y * (ONED ? n0 : 2 * n0) * W;
    auto spec = [&](int k, int r) -> V {
        V y = C[(size_t)k * cst + r];
        if constexpr (ONED) {
            y.x = y.x * y.x + y.y * y.y;
            y.y = T(0);
        }
        return y;
    };
    auto cvt = [](double2 d) -> V {
        V v;
        v.x = (T)d.x;
        v.y = (T)d.y;
        return v;
    };
    // Z[k] = (Y[k] + conj Y[Hp-k]) + i W^-k (Y[k] - conj Y[Hp-k]); rows fastest
    // (BLUE: times the chirp, zero-padded to M)
    FcgIdx it(threadIdx.x, blockDim.x, rpb);
    for (int idx = threadIdx.x; idx < rpb * NF; idx += blockDim.x, it.next()) {
        const int k = it.a, rr = it.b, r = r0 + rr;
        V z = cx_zero<V>();
        if (r < rows && k < Hp) {
            V yk = spec(k, r), yc = cx_conj(spec(Hp - k, r));
            if (k == 0) {
                yk.y = T(0);
                yc.y = T(0);
            }
            const V e = cx_add(yk, yc), d = cx_sub(yk, yc);
            const double2 wdd = __ldg(&twl1[k]);
            V w;
            w.x = (T)wdd.x;
            w.y = (T)-wdd.y;
            const V wd = cx_mul(w, d);
            z.x = e.x - wd.y;
            z.y = e.y + wd.x;
            if constexpr (BLUE) z = cx_mul(z, cvt(__ldg(&chirp[k])));
        }
        S[fcg_slot<V>(rr, k, stride)] = z;
    }
    __syncthreads();
    const V *Z;
    if constexpr (BLUE) {
        V *F = fcg_fft<V, false>(S, S2, stride, rad, rpb, twm, NF, FcNoLoad<V>{}, false);
        for (int idx = threadIdx.x; idx < rpb * NF; idx += blockDim.x) {
            const int rr = idx / NF, i = idx - rr * NF;
            V &v = F[fcg_slot<V>(rr, i, stride)];
            v = cx_mul(v, cvt(__ldg(&Bf[i])));
        }
        __syncthreads();
        Z = fcg_fft<V, true>(F, F == S ? S2 : S, stride, rad, rpb, twm, NF, FcNoLoad<V>{}, false);
    } else {
        Z = fcg_fft<V, true>(S, S2, stride, rad, rpb, twl1, L1, FcNoLoad<V>{}, false);
    }
    const T scale = T(1) / (T)L1;
    auto val = [&](int rr, int c) -> T {
        V z = Z[fcg_slot<V>(rr, c >> 1, stride)];
        if constexpr (BLUE) z = cx_mul(z, cvt(__ldg(&chirp[c >> 1])));
        return ((c & 1) ? z.y : z.x) * scale;
    };
    auto put = [&](int i, int j, T y) {
        const size_t o = (size_t)i * W + j;
        if (mode == 0 || mode == 1) {
            const T cn = norm[ONED ? (size_t)j : o];
            y = mode == 0 ? (cn < threshold ? T(NAN) : y / cn) : (cn > threshold ? y / cn : T(0));
        } else if (mode == 2) {
            const T cn = (T)((int64_t)(ONED ? 1 : n0 - abs(i - n0)) * (n1 - abs(j - n1)));
            y = cn < threshold ? T(NAN) : y / cn;
        }
        out[o] = y;
    };
    FcgIdx ot(threadIdx.x, blockDim.x, W);
    for (int idx = threadIdx.x; idx < rpb * W; idx += blockDim.x, ot.next()) {
        const int rr = ot.a, j = ot.b, r = r0 + rr;
        if (r >= rows) continue;
        // |j - n1| <= n1 <= L1 / 2: one conditional add gives the residue
        const int c = j - n1 < 0 ? j - n1 + L1 : j - n1;
        if constexpr (ONED) {
            put(r, j, val(rr, c));
        } else {
            if (r < n0) put(n0 + r, j, val(rr, c));
            if (r > 0) put(n0 - r, j, val(rr, n1 - j < 0 ? n1 - j + L1 : n1 - j));
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
    if (ndim == 2 && batch * 2 * (int64_t)n[0] <= 65535) {
        const dim3 grid((unsigned)std::min<int64_t>((2 * (int64_t)n[1] + 255) / 256, 64),
                        (unsigned)(batch * 2 * n[0]));
        if (dtype == IDIWF_F64)
            crop2d_kernel<double><<<grid, 256, 0, stream>>>(static_cast<const double *>(full), g[0], g[1], n[0], n[1],
                                                            static_cast<const double *>(norm), mode, threshold,
                                                            static_cast<double *>(out));
        else if (dtype == IDIWF_F32)
            crop2d_kernel<float><<<grid, 256, 0, stream>>>(static_cast<const float *>(full), g[0], g[1], n[0], n[1],
                                                           static_cast<const float *>(norm), mode, (float)threshold,
                                                           static_cast<float *>(out));
        else
            return set_error(IDIWF_ERR_INVALID_ARGUMENT, "dtype must be IDIWF_F64 or IDIWF_F32");
        IDIWF_CUDA_CHECK(cudaGetLastError());
        return IDIWF_OK;
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

// Workspace of idiwf_fft_autocorr: the twiddle table, then T and C of one
// group of images, each 256-byte aligned.
static size_t fc_align(size_t b) { return (b + 255) & ~(size_t)255; }
static bool fc_pow2(int v) { return v >= 4 && v <= 4096 && (v & (v - 1)) == 0; }
static int fc_log2(int v) {
    int l = 0;
    while ((1 << l) < v) ++l;
    return l;
}
struct FcPlan {
    int n0, n1, H, G0, G1, N, logh, logg0;
    int rpb, cpb;         // rows per block (passes A and C), columns per block (pass B)
    size_t vsz;           // bytes per complex value
    size_t t_img, c_img;  // complex values of T and C per image
    size_t tw_bytes, t_bytes, c_bytes;
    int64_t group;        // images per launch
};
// Images per launch: all of them while T and C of the group stay within
// 256 MB, else equal groups under that.
static FcPlan fc_plan(int64_t batch, int n0, int n1, int dtype) {
    FcPlan p{};
    p.n0 = n0;
    p.n1 = n1;
    p.H = n1;
    p.G0 = 2 * n0;
    p.G1 = 2 * n1;
    p.N = std::max(p.G0, p.G1);
    p.logh = fc_log2(p.H);
    p.logg0 = fc_log2(p.G0);
    p.vsz = dtype == IDIWF_F64 ? 16 : 8;
    p.rpb = std::max(1, std::min(kFcBlockElems / p.H, n0));
    p.cpb = std::max(1, std::min(kFcBlockElems / p.G0, 1 << fc_log2(p.H + 1)));
    p.t_img = (size_t)(p.H + 1) * n0;
    p.c_img = (size_t)(p.H + 1) * (n0 + 1);
    p.tw_bytes = fc_align((size_t)p.N * sizeof(double2));
    const size_t per = (p.t_img + p.c_img) * p.vsz;
    const int64_t gmax = std::max<int64_t>(1, std::min<int64_t>(65535, (int64_t)((256u << 20) / per)));
    const int64_t ngroups = (std::max<int64_t>(batch, 1) + gmax - 1) / gmax;
    p.group = (std::max<int64_t>(batch, 1) + ngroups - 1) / ngroups;
    p.t_bytes = fc_align(p.t_img * p.vsz * p.group);
    p.c_bytes = fc_align(p.c_img * p.vsz * p.group);
    return p;
}

// ---- general lengths: host side ----
// Smallest N >= x whose prime factors are 2, 3, 5, 7, 11 (the reference's
// idi.util.fastlen).
static int fcg_fastlen(int x) {
    for (int n = std::max(1, x);; ++n) {
        int m = n;
        for (int f : {2, 3, 5, 7, 11})
            while (m % f == 0) m /= f;
        if (m == 1) return n;
    }
}
// Radices of n (11, 7, 5, 3, then 8s, then 4 or 2); false if n has another
// prime factor or needs too many passes.
static bool fcg_radices(int n, FcgRad &rad) {
    rad = FcgRad{};
    rad.n = n;
    int m = n;
    for (int f : {11, 7, 5, 3})
        while (m % f == 0) {
            if (rad.np == kFcgMaxPasses) return false;
            rad.r[rad.np++] = f;
            m /= f;
        }
    while (m % 8 == 0 && m > 1) {
        if (rad.np == kFcgMaxPasses) return false;
        rad.r[rad.np++] = 8;
        m /= 8;
    }
    if (m == 2 || m == 4) {
        if (rad.np == kFcgMaxPasses) return false;
        rad.r[rad.np++] = m;
        m = 1;
    }
    return m == 1;
}
// Threads of a general-path block holding `values` complex values in
// `smem` bytes (every pass loops over its butterflies, so any count works):
// 256 where two or more blocks fit in an SM's shared memory, else 512 (more
// warps per SM either way), fewer for small blocks.
static int fcg_threads(int values, size_t smem, size_t vsz) {
    // FP32 (8-byte values): at most 256, the kernels' launch bound
    const int cap = (2 * smem <= 227 * 1024 || vsz == 8) ? 256 : 512;
    return std::min(cap, std::max(32, (values / 4 + 31) / 32 * 32));
}
constexpr int kFcgMaxLen = 4096;  // G0, G1 and L1 of the general path
static int fcg_stride(int n, int lkc) { return n + ((n - 1) >> lkc) + 1; }

struct FcgPlan {
    int n0, n1, G0, G1, L1, m, Hp;
    int ppb, cpb, rpb;  // row pairs (pass A), columns (B), rows (C) per block
    FcgRad radA, radB, radC;  // radC: Hp, or M with blue
    int thrA, thrB, thrC, strA, strB, strC;
    size_t vsz, t_img, c_img;
    size_t twA_bytes, twB_bytes, twC_bytes, blue_bytes, t_bytes, c_bytes;
    int64_t group;
    bool oned;  // n0 independent lines: no column pass, no C
    bool blue;  // odd G1: the inverse of Hp = (G1 - 1) / 2 values by Bluestein
    int M;      // Bluestein's FFT length
};
static bool fcg_plan(int64_t batch, int n0, int n1, int dtype, FcgPlan &p, bool oned = false) {
    if (n0 < 1 || n1 < 1 || (!oned && n0 > kFcgMaxLen) || n1 > kFcgMaxLen) return false;
    p = FcgPlan{};
    p.oned = oned;
    p.n0 = n0;
    p.n1 = n1;
    p.G0 = fcg_fastlen(2 * n0);
    p.G1 = fcg_fastlen(2 * n1);
    // numpy's irfftn default along the last axis: 2 (G1/2 + 1 - 1) values
    p.L1 = p.G1 % 2 ? p.G1 - 1 : p.G1;
    p.m = p.G1 / 2 + 1;
    p.Hp = p.L1 / 2;
    if (p.G0 > kFcgMaxLen || p.G1 > kFcgMaxLen) return false;
    if (oned) p.G0 = 1;  // no column pass
    if (!fcg_radices(p.G1, p.radA)) return false;
    if (!oned && !fcg_radices(p.G0, p.radB)) return false;
    p.blue = !fcg_radices(p.Hp, p.radC);
    if (p.blue) {
        // the shortest smooth length: measured faster than longer lengths with
        // cheaper radices (2304 or 640 instead of 2079 or 605)
        p.M = fcg_fastlen(2 * p.Hp - 1);
        if (p.M > kFcgMaxLen || !fcg_radices(p.M, p.radC)) return false;
    }
    const int nC = p.radC.n;  // values per row in pass C
    p.vsz = dtype == IDIWF_F64 ? 16 : 8;
    const int lkc = p.vsz == 16 ? 3 : 4;
    // values per block: 2048 in FP64 (three blocks per SM with ping-pong
    // buffers; measured 2-11 % faster than 4096 despite unpaired inverses
    // for columns above 1024), 4096 in FP32
    const int be = p.vsz == 16 ? 2048 : kFcBlockElems;
    p.ppb = std::max(1, std::min(be / p.G1, (n0 + 1) / 2));
    p.cpb = std::max(1, std::min(be / p.G0, p.m));
    p.rpb = std::max(1, std::min(be / nC, oned ? n0 : n0 + 1));
    p.strA = fcg_stride(p.G1, lkc);
    p.strB = fcg_stride(p.G0, lkc);
    p.strC = fcg_stride(nC, lkc);
    // ping-pong buffers of count sequences each
    p.thrA = fcg_threads(p.ppb * p.G1, 2 * (size_t)p.ppb * p.strA * p.vsz, p.vsz);
    p.thrB = fcg_threads(p.cpb * p.G0, 2 * (size_t)p.cpb * p.strB * p.vsz, p.vsz);
    p.thrC = fcg_threads(p.rpb * nC, 2 * (size_t)p.rpb * p.strC * p.vsz, p.vsz);
    p.t_img = (size_t)p.m * n0;
    p.c_img = oned ? 0 : (size_t)p.m * (n0 + 1);
    p.twA_bytes = fc_align((size_t)p.G1 * sizeof(double2));
    p.twB_bytes = oned ? 0 : fc_align((size_t)p.G0 * sizeof(double2));
    p.twC_bytes = fc_align((size_t)p.L1 * sizeof(double2));
    // chirp (Hp), filter spectrum (M), twiddles of M
    p.blue_bytes = p.blue ? fc_align((size_t)p.Hp * sizeof(double2)) + 2 * fc_align((size_t)p.M * sizeof(double2)) : 0;
    const size_t per = (p.t_img + p.c_img) * p.vsz;
    const int64_t gmax = std::max<int64_t>(1, std::min<int64_t>(65535, (int64_t)((256u << 20) / per)));
    const int64_t ngroups = (std::max<int64_t>(batch, 1) + gmax - 1) / gmax;
    p.group = (std::max<int64_t>(batch, 1) + ngroups - 1) / ngroups;
    p.t_bytes = fc_align(p.t_img * p.vsz * p.group);
    p.c_bytes = fc_align(p.c_img * p.vsz * p.group);
    return true;
}
// For an odd G1 the reference's inverse has G1 - 1 values and its pair count
// (the same transform of ones) is not the closed form of mode 2.
static const char *const kFcOddPairs =
    "mode 2 (closed-form pair count) does not hold for an odd fastlen(2 n1); transform ones with mode -1 and pass "
    "the result as norm with mode 0";
static size_t fcg_ws_bytes(const FcgPlan &p) {
    return p.twA_bytes + p.twB_bytes + p.twC_bytes + p.blue_bytes + p.t_bytes + p.c_bytes;
}

template <typename T>
static idiwf_status fcg_run(const T *x, int64_t batch, const FcgPlan &p, const T *norm, int mode, double threshold,
                            T *out, unsigned char *ws, cudaStream_t stream) {
    using V = typename Cx<T>::t;
    double2 *twA = reinterpret_cast<double2 *>(ws);
    double2 *twB = reinterpret_cast<double2 *>(ws + p.twA_bytes);
    double2 *twC = reinterpret_cast<double2 *>(ws + p.twA_bytes + p.twB_bytes);
    unsigned char *bl = ws + p.twA_bytes + p.twB_bytes + p.twC_bytes;
    double2 *chirp = p.blue ? reinterpret_cast<double2 *>(bl) : nullptr;
    double2 *Bf = p.blue ? reinterpret_cast<double2 *>(bl + fc_align((size_t)p.Hp * sizeof(double2))) : nullptr;
    double2 *twM = p.blue ? Bf + fc_align((size_t)p.M * sizeof(double2)) / sizeof(double2) : nullptr;
    unsigned char *rest = bl + p.blue_bytes;
    V *Tt = reinterpret_cast<V *>(rest);
    V *C = reinterpret_cast<V *>(rest + p.t_bytes);
    fc_twiddle_kernel<<<(p.G1 + 255) / 256, 256, 0, stream>>>(twA, p.G1);
    if (!p.oned) fc_twiddle_kernel<<<(p.G0 + 255) / 256, 256, 0, stream>>>(twB, p.G0);
    fc_twiddle_kernel<<<(p.L1 + 255) / 256, 256, 0, stream>>>(twC, p.L1);
    IDIWF_CUDA_CHECK(cudaGetLastError());
    if (p.blue) {
        fc_twiddle_kernel<<<(p.M + 255) / 256, 256, 0, stream>>>(twM, p.M);
        fcg_chirp_kernel<<<(p.Hp + 255) / 256, 256, 0, stream>>>(chirp, p.Hp);
        const int strM = fcg_stride(p.M, 3);  // the filter is made in FP64
        const size_t smF = 2 * (size_t)strM * sizeof(double2);
        IDIWF_CUDA_CHECK(
            cudaFuncSetAttribute(fcg_blue_filter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smF));
        fcg_blue_filter_kernel<<<1, 512, smF, stream>>>(chirp, p.Hp, p.radC, strM, twM, Bf);
        IDIWF_CUDA_CHECK(cudaGetLastError());
    }
    const size_t smA = 2 * (size_t)p.ppb * p.strA * sizeof(V), smB = 2 * (size_t)p.cpb * p.strB * sizeof(V);
    const size_t smC = 2 * (size_t)p.rpb * p.strC * sizeof(V);
    IDIWF_CUDA_CHECK(cudaFuncSetAttribute(fcg_rows_fwd<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smA));
    if (!p.oned)
        IDIWF_CUDA_CHECK(cudaFuncSetAttribute(fcg_cols<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smB));
    void *kC = p.oned ? (p.blue ? (void *)fcg_rows_inv<T, true, true> : (void *)fcg_rows_inv<T, true, false>)
                      : (p.blue ? (void *)fcg_rows_inv<T, false, true> : (void *)fcg_rows_inv<T, false, false>);
    IDIWF_CUDA_CHECK(cudaFuncSetAttribute(kC, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smC));
    const int npairs = (p.n0 + 1) / 2;
    const unsigned blkA = (unsigned)((npairs + p.ppb - 1) / p.ppb), blkB = (unsigned)((p.m + p.cpb - 1) / p.cpb);
    const int rowsC = p.oned ? p.n0 : p.n0 + 1;
    const unsigned blkC = (unsigned)((rowsC + p.rpb - 1) / p.rpb);
    const size_t in_img = (size_t)p.n0 * p.n1, out_img = (size_t)(p.oned ? p.n0 : 2 * p.n0) * (2 * p.n1);
    for (int64_t b0 = 0; b0 < batch; b0 += p.group) {
        const unsigned g = (unsigned)std::min<int64_t>(p.group, batch - b0);
        fcg_rows_fwd<T><<<dim3(blkA, g), p.thrA, smA, stream>>>(x + b0 * in_img, p.n0, p.n1, p.ppb, p.radA, p.strA,
                                                                  twA, p.m, Tt, p.t_img);
        if (!p.oned)
            fcg_cols<T><<<dim3(blkB, g), p.thrB, smB, stream>>>(Tt, p.t_img, p.n0, p.m, p.cpb, p.radB, p.strB, twB,
                                                                  C, p.c_img);
        IDIWF_CUDA_CHECK(cudaGetLastError());
        const V *Csrc = p.oned ? Tt : C;
        const size_t c_img = p.oned ? p.t_img : p.c_img;
        T *o = out + b0 * out_img;
        T thr = (T)threshold;
        void *args[] = {(void *)&Csrc, (void *)&c_img, (void *)&p.n0, (void *)&p.n1, (void *)&p.Hp, (void *)&p.rpb,
                        (void *)&p.radC, (void *)&p.strC, (void *)&twC, (void *)&twM, (void *)&chirp, (void *)&Bf,
                        (void *)&norm, (void *)&mode, (void *)&thr, (void *)&o};
        IDIWF_CUDA_CHECK(cudaLaunchKernel(kC, dim3(blkC, g), dim3(p.thrC), args, smC, stream));
    }
    return IDIWF_OK;
}

extern "C" size_t idiwf_fft_autocorr_workspace_size(int64_t batch, int32_t n0, int32_t n1, int32_t dtype) {
    if (batch <= 0 || (dtype != IDIWF_F64 && dtype != IDIWF_F32)) return 0;
    if (fc_pow2(n0) && fc_pow2(n1)) {
        const FcPlan p = fc_plan(batch, n0, n1, dtype);
        return p.tw_bytes + p.t_bytes + p.c_bytes;
    }
    FcgPlan g;
    if (!fcg_plan(batch, n0, n1, dtype, g)) return 0;
    return fcg_ws_bytes(g);
}

template <typename T, int EA, int EB>
static idiwf_status fc_launch(const T *x, int64_t batch, const FcPlan &p, const T *norm, int mode, double threshold,
                              T *out, const double2 *tw, typename Cx<T>::t *Tt, typename Cx<T>::t *C,
                              cudaStream_t stream) {
    using V = typename Cx<T>::t;
    const int thrA = std::max(1, p.rpb * p.H / EA), thrB = std::max(1, p.cpb * p.G0 / EB);
    const size_t smA = fc_smem_values<V>(p.rpb, p.logh, fc_rows_swz<V>(p.logh, p.rpb)) * sizeof(V);
    const size_t smB = fc_smem_values<V>(p.cpb, p.logg0, FcSwz{31, 0}) * sizeof(V);
    IDIWF_CUDA_CHECK(cudaFuncSetAttribute(fc_rows_fwd<T, EA>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smA));
    IDIWF_CUDA_CHECK(cudaFuncSetAttribute(fc_rows_inv<T, EA>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smA));
    IDIWF_CUDA_CHECK(cudaFuncSetAttribute(fc_cols<T, EB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smB));
    const unsigned blkA = (unsigned)((p.n0 + p.rpb - 1) / p.rpb), blkC = (unsigned)((p.n0 + 1 + p.rpb - 1) / p.rpb);
    const unsigned blkB = (unsigned)((p.H + 1 + p.cpb - 1) / p.cpb);
    const size_t in_img = (size_t)p.n0 * p.n1, out_img = (size_t)p.G0 * p.G1;
    for (int64_t b0 = 0; b0 < batch; b0 += p.group) {
        const unsigned g = (unsigned)std::min<int64_t>(p.group, batch - b0);
        fc_rows_fwd<T, EA><<<dim3(blkA, g), thrA, smA, stream>>>(x + b0 * in_img, p.n0, p.n1, p.logh, p.rpb, tw, p.N,
                                                                    Tt, p.t_img);
        fc_cols<T, EB><<<dim3(blkB, g), thrB, smB, stream>>>(Tt, p.t_img, p.n0, p.H + 1, p.logg0, p.cpb, tw, p.N, C,
                                                             p.c_img);
        fc_rows_inv<T, EA><<<dim3(blkC, g), thrA, smA, stream>>>(C, p.c_img, p.n0, p.n1, p.logh, p.rpb, tw, p.N, norm,
                                                                    mode, (T)threshold, out + b0 * out_img);
        IDIWF_CUDA_CHECK(cudaGetLastError());
    }
    return IDIWF_OK;
}

template <typename T>
static idiwf_status fc_run(const T *x, int64_t batch, const FcPlan &p, const T *norm, int mode, double threshold,
                           T *out, unsigned char *ws, cudaStream_t stream) {
    using V = typename Cx<T>::t;
    double2 *tw = reinterpret_cast<double2 *>(ws);
    V *Tt = reinterpret_cast<V *>(ws + p.tw_bytes);
    V *C = reinterpret_cast<V *>(ws + p.tw_bytes + p.t_bytes);
    fc_twiddle_kernel<<<(p.N + 255) / 256, 256, 0, stream>>>(tw, p.N);
    IDIWF_CUDA_CHECK(cudaGetLastError());
    if constexpr (sizeof(T) == 4) {
        return fc_launch<T, 16, 16>(x, batch, p, norm, mode, threshold, out, tw, Tt, C, stream);
    } else {
        if (p.G0 > kFcBlockElems)  // one 8192-point column per block: 16 values per thread keep it at 512 threads
            return fc_launch<T, 8, 16>(x, batch, p, norm, mode, threshold, out, tw, Tt, C, stream);
        return fc_launch<T, 8, 8>(x, batch, p, norm, mode, threshold, out, tw, Tt, C, stream);
    }
}

extern "C" idiwf_status idiwf_fft_autocorr(const void *x, int32_t dtype, int64_t batch, int32_t n0, int32_t n1,
                                           const void *norm, int32_t mode, double threshold, void *out,
                                           void *workspace, size_t workspace_bytes, cudaStream_t stream) {
    if (!x || !out) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "NULL argument");
    if (batch <= 0) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "batch must be positive");
    if ((dtype == IDIWF_F64 || dtype == IDIWF_F32) && idiwf_fft_autocorr_workspace_size(batch, n0, n1, dtype) == 0)
        return set_error(IDIWF_ERR_UNSUPPORTED,
                         "shape not supported by the hand-written autocorrelation (powers of two from 4 to 4096, or "
                         "fastlen(2 n0), fastlen(2 n1) <= 4096)");
    if (mode < -1 || mode > 2) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "mode must be -1, 0, 1 or 2");
    if ((mode == 0 || mode == 1) && !norm) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "modes 0 and 1 need norm");
    const size_t need = idiwf_fft_autocorr_workspace_size(batch, n0, n1, dtype);
    if (need == 0) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "dtype must be IDIWF_F64 or IDIWF_F32");
    if (!workspace || workspace_bytes < need)
        return set_error(IDIWF_ERR_WORKSPACE, "workspace smaller than idiwf_fft_autocorr_workspace_size()");
    if (reinterpret_cast<uintptr_t>(workspace) & 255)
        return set_error(IDIWF_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    if (!(fc_pow2(n0) && fc_pow2(n1))) {
        FcgPlan g;
        fcg_plan(batch, n0, n1, dtype, g);
        if (g.blue && mode == 2)
            return set_error(IDIWF_ERR_UNSUPPORTED, kFcOddPairs);
        if (dtype == IDIWF_F64)
            return fcg_run<double>(static_cast<const double *>(x), batch, g, static_cast<const double *>(norm), mode,
                                   threshold, static_cast<double *>(out), ws, stream);
        return fcg_run<float>(static_cast<const float *>(x), batch, g, static_cast<const float *>(norm), mode,
                              threshold, static_cast<float *>(out), ws, stream);
    }
    // power-of-two shapes: rows are read and written as pairs of values
    const uintptr_t pair = dtype == IDIWF_F64 ? 15 : 7;
    if ((reinterpret_cast<uintptr_t>(x) & pair) || (reinterpret_cast<uintptr_t>(out) & pair))
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "x and out must be aligned to two elements");
    const FcPlan p = fc_plan(batch, n0, n1, dtype);
    if (dtype == IDIWF_F64)
        return fc_run<double>(static_cast<const double *>(x), batch, p, static_cast<const double *>(norm), mode,
                              threshold, static_cast<double *>(out), ws, stream);
    return fc_run<float>(static_cast<const float *>(x), batch, p, static_cast<const float *>(norm), mode, threshold,
                         static_cast<float *>(out), ws, stream);
}

// ---- 1D: independent lines ----
// Lines run as images of kFc1dLines rows (plus one image of the remainder).
constexpr int kFc1dLines = 1024;
static bool fc1d_plans(int64_t lines, int n, int dtype, FcgPlan &full, FcgPlan &rest, int64_t &nfull, int &nrest) {
    if (lines <= 0 || (dtype != IDIWF_F64 && dtype != IDIWF_F32)) return false;
    const int L = (int)std::min<int64_t>(lines, kFc1dLines);
    nfull = lines / L;
    nrest = (int)(lines - nfull * L);
    if (!fcg_plan(nfull, L, n, dtype, full, true)) return false;
    if (nrest && !fcg_plan(1, nrest, n, dtype, rest, true)) return false;
    return true;
}

extern "C" size_t idiwf_fft_autocorr_1d_workspace_size(int64_t lines, int32_t n, int32_t dtype) {
    FcgPlan full, rest;
    int64_t nfull;
    int nrest;
    if (!fc1d_plans(lines, n, dtype, full, rest, nfull, nrest)) return 0;
    // the remainder image reuses the same workspace (it is smaller)
    return fcg_ws_bytes(full);
}

extern "C" idiwf_status idiwf_fft_autocorr_1d(const void *x, int32_t dtype, int64_t lines, int32_t n,
                                              const void *norm, int32_t mode, double threshold, void *out,
                                              void *workspace, size_t workspace_bytes, cudaStream_t stream) {
    if (!x || !out) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "NULL argument");
    if (lines <= 0) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "lines must be positive");
    if (dtype != IDIWF_F64 && dtype != IDIWF_F32)
        return set_error(IDIWF_ERR_INVALID_ARGUMENT, "dtype must be IDIWF_F64 or IDIWF_F32");
    FcgPlan full, rest;
    int64_t nfull;
    int nrest;
    if (!fc1d_plans(lines, n, dtype, full, rest, nfull, nrest))
        return set_error(IDIWF_ERR_UNSUPPORTED,
                         "length not supported by the hand-written autocorrelation (fastlen(2 n) <= 4096)");
    if (full.blue && mode == 2) return set_error(IDIWF_ERR_UNSUPPORTED, kFcOddPairs);
    if (mode < -1 || mode > 2) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "mode must be -1, 0, 1 or 2");
    if ((mode == 0 || mode == 1) && !norm) return set_error(IDIWF_ERR_INVALID_ARGUMENT, "modes 0 and 1 need norm");
    const size_t need = idiwf_fft_autocorr_1d_workspace_size(lines, n, dtype);
    if (!workspace || workspace_bytes < need)
        return set_error(IDIWF_ERR_WORKSPACE, "workspace smaller than idiwf_fft_autocorr_1d_workspace_size()");
    if (reinterpret_cast<uintptr_t>(workspace) & 255)
        return set_error(IDIWF_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    const size_t es = dtype == IDIWF_F64 ? 8 : 4;
    const int64_t done = nfull * full.n0;
    const unsigned char *xb = static_cast<const unsigned char *>(x);
    unsigned char *ob = static_cast<unsigned char *>(out);
    for (int part = 0; part < 2; ++part) {
        const FcgPlan &p = part == 0 ? full : rest;
        const int64_t images = part == 0 ? nfull : (nrest ? 1 : 0);
        if (images == 0) continue;
        const void *xp = xb + (part == 0 ? 0 : (size_t)done * n * es);
        void *op = ob + (part == 0 ? 0 : (size_t)done * 2 * n * es);
        idiwf_status st;
        if (dtype == IDIWF_F64)
            st = fcg_run<double>(static_cast<const double *>(xp), images, p, static_cast<const double *>(norm), mode,
                                 threshold, static_cast<double *>(op), ws, stream);
        else
            st = fcg_run<float>(static_cast<const float *>(xp), images, p, static_cast<const float *>(norm), mode,
                                threshold, static_cast<float *>(op), ws, stream);
        if (st != IDIWF_OK) return st;
    }
    return IDIWF_OK;
}
