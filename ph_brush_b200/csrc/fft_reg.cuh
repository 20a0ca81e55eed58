// Register-resident DFTs of compile-time length for the mesh kernels (sm_100a).
//
// rdft<N, S>(v) transforms N complex values held in registers in place:
// v[k] <- sum_j v[j] exp(S 2 pi i j k / N), S = -1 forward, +1 inverse
// (unnormalised).  Mixed radix 4/2/3/5, decimation in time; every index and
// twiddle is a compile-time constant, so the butterflies are straight-line
// FMAs on registers.  The twiddle constants are computed at compile time in
// double precision (Taylor series of sin and cos after reduction to
// (-pi, pi]) and rounded once to float.
#pragma once
#include <cuda_runtime.h>
#include "fft.cuh"

// unrolled in device code (the host pass of these __host__ __device__ functions is for tests)
#if defined(__CUDA_ARCH__)
#define RFFT_UNROLL _Pragma("unroll")
#else
#define RFFT_UNROLL
#endif

namespace rfft {

constexpr double kPi = 3.14159265358979323846264338327950288;

constexpr double taylor_sin(double x) {
    double x2 = x * x, t = x, s = x;
    for (int i = 1; i < 16; ++i) { t *= -x2 / ((2.0 * i) * (2.0 * i + 1.0)); s += t; }
    return s;
}
constexpr double taylor_cos(double x) {
    double x2 = x * x, t = 1.0, s = 1.0;
    for (int i = 1; i < 16; ++i) { t *= -x2 / ((2.0 * i - 1.0) * (2.0 * i)); s += t; }
    return s;
}
// values within 1e-14 of 0, +-1/2 or +-1 are snapped to them (the Taylor sums miss them by ~1e-16)
constexpr double snap(double v) {
    const double k[5] = {0.0, 0.5, -0.5, 1.0, -1.0};
    for (double c : k)
        if (v - c < 1e-14 && c - v < 1e-14) return c;
    return v;
}
// cos and sin of 2 pi j / n
constexpr double cos2pi(long j, long n) {
    j %= n; if (j < 0) j += n; if (2 * j > n) j -= n;
    return snap(taylor_cos(2.0 * kPi * (double)j / (double)n));
}
constexpr double sin2pi(long j, long n) {
    j %= n; if (j < 0) j += n; if (2 * j > n) j -= n;
    return snap(taylor_sin(2.0 * kPi * (double)j / (double)n));
}

template <int N>
struct Tw {
    float c[N], s[N];
    constexpr Tw() : c(), s() {
        for (int j = 0; j < N; ++j) { c[j] = (float)cos2pi(j, N); s[j] = (float)sin2pi(j, N); }
    }
};

// a * (c + i s)
__host__ __device__ __forceinline__ float2 cmulc(float2 a, float c, float s) {
    return make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
}

template <int N, int S>
__host__ __device__ __forceinline__ void rdft(float2 (&v)[N]) {
    static_assert(S == 1 || S == -1, "sign");
    constexpr float sg = (float)S;
    if constexpr (N == 1) {
    } else if constexpr (N == 2) {
        const float2 a = v[0], b = v[1];
        v[0] = cadd(a, b); v[1] = csub(a, b);
    } else if constexpr (N == 3) {
        const float s3 = 0.86602540378443864676f;
        const float2 s = cadd(v[1], v[2]), dd = cmul_si(csub(v[1], v[2]), sg * s3);
        const float2 m = csub(v[0], cscale(s, 0.5f));
        v[0] = cadd(v[0], s); v[1] = cadd(m, dd); v[2] = csub(m, dd);
    } else if constexpr (N == 4) {
        const float2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
        const float2 c = cadd(v[1], v[3]), dd = cmul_si(csub(v[1], v[3]), sg);
        v[0] = cadd(a, c); v[2] = csub(a, c); v[1] = cadd(b, dd); v[3] = csub(b, dd);
    } else if constexpr (N == 5) {
        dft_radix(v, 5, sg);
    } else {
        // N = R * M: length-M DFTs of the R decimated sequences v[R m + r], twiddle W_N^(r k),
        // then length-R DFTs across r: X[k + M q] = sum_r W_R^(r q) W_N^(r k) Y_r[k]
        constexpr int R = (N % 4 == 0) ? 4 : (N % 2 == 0) ? 2 : (N % 3 == 0) ? 3 : 5;
        constexpr int M = N / R;
        static_assert(R * M == N, "length must be 2^a 3^b 5^c");
        constexpr Tw<N> T{};
        float2 sub[R][M];
RFFT_UNROLL
        for (int r = 0; r < R; ++r) {
RFFT_UNROLL
            for (int m = 0; m < M; ++m) sub[r][m] = v[R * m + r];
            rdft<M, S>(sub[r]);
        }
RFFT_UNROLL
        for (int k = 0; k < M; ++k) {
            float2 t[R];
            t[0] = sub[0][k];
RFFT_UNROLL
            for (int r = 1; r < R; ++r) t[r] = cmulc(sub[r][k], T.c[r * k], sg * T.s[r * k]);
            rdft<R, S>(t);
RFFT_UNROLL
            for (int q = 0; q < R; ++q) v[k + M * q] = t[q];
        }
    }
}

}  // namespace rfft
