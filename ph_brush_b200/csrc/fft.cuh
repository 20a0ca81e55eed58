// Shared-memory FFT building blocks used by the mesh kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>

// ---------------------------------------------------------------------------
// Mixed-radix Stockham autosort FFT over `nlines` lines held in shared memory
// (Govindaraju et al., "High performance discrete Fourier transforms on
// graphics processors", SC'08).  Element e of line l lives at l*ls + e*es.
// Returns the buffer that holds the result (a or b).
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by sign*i
__host__ __device__ __forceinline__ float2 cmul_si(float2 a, float sign) { return make_float2(-sign * a.y, sign * a.x); }

__host__ __device__ __forceinline__ void dft_radix(float2* v, int R, float sign) {
    if (R == 2) {
        float2 a = v[0], b = v[1];
        v[0] = cadd(a, b); v[1] = csub(a, b);
    } else if (R == 4) {
        float2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
        float2 c = cadd(v[1], v[3]), d = cmul_si(csub(v[1], v[3]), sign);
        v[0] = cadd(a, c); v[2] = csub(a, c); v[1] = cadd(b, d); v[3] = csub(b, d);
    } else if (R == 3) {
        const float s3 = 0.86602540378443864676f;
        float2 s = cadd(v[1], v[2]), d = cmul_si(csub(v[1], v[2]), sign * s3);
        float2 m = csub(v[0], cscale(s, 0.5f));
        v[0] = cadd(v[0], s); v[1] = cadd(m, d); v[2] = csub(m, d);
    } else {  // R == 5
        const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;
        const float s1 = 0.95105651629515357212f, s2 = 0.58778525229247312917f;
        float2 a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
        float2 a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
        float2 r1 = cadd(v[0], cadd(cscale(a1, c1), cscale(a2, c2)));
        float2 r2 = cadd(v[0], cadd(cscale(a1, c2), cscale(a2, c1)));
        float2 i1 = cmul_si(cadd(cscale(b1, s1), cscale(b2, s2)), sign);
        float2 i2 = cmul_si(csub(cscale(b1, s2), cscale(b2, s1)), sign);
        v[0] = cadd(v[0], cadd(a1, a2));
        v[1] = cadd(r1, i1); v[4] = csub(r1, i1);
        v[2] = cadd(r2, i2); v[3] = csub(r2, i2);
    }
}

__device__ __forceinline__ int fft_plan(int n, int* rad) {
    int ns = 0, m = n;
    while (m % 4 == 0) { rad[ns++] = 4; m /= 4; }
    if (m % 2 == 0) { rad[ns++] = 2; m /= 2; }
    while (m % 3 == 0) { rad[ns++] = 3; m /= 3; }
    while (m % 5 == 0) { rad[ns++] = 5; m /= 5; }
    return ns;
}

// a / b and a % b for 0 <= a < 2^22 through a float reciprocal of b, corrected to exact.
struct FastDiv {
    int b;
    float rb;
    __device__ __forceinline__ explicit FastDiv(int b_) : b(b_), rb(1.0f / (float)b_) {}
    __device__ __forceinline__ int div(int a, int& rem) const {
        int q = __float2int_rz((float)a * rb);
        int r = a - q * b;
        if (r < 0) { --q; r += b; } else if (r >= b) { ++q; r -= b; }
        rem = r;
        return q;
    }
};

// One Stockham stage of radix R over all lines (R is a compile-time constant, so
// the butterfly's R values stay in registers).
template <int R, int NT>
__device__ __forceinline__ void fft_stage(const float2* __restrict__ a, float2* __restrict__ b, int n, int nlines, int ls,
                                          int es, const float2* __restrict__ tw, float sign, bool line_fastest, int Ns,
                                          const FastDiv& dl) {
    const int nb = n / R;
    const int tstride = n / (Ns * R);
    const int total = nb * nlines;
    const FastDiv dnb(nb), dns(Ns);
    for (int t = threadIdx.x; t < total; t += NT) {
        int line, j, k;
        if (line_fastest) j = dl.div(t, line);
        else line = dnb.div(t, j);
        const int jq = dns.div(j, k);
        float2 v[R];
        const float2* src = a + line * ls;
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = src[(j + r * nb) * es];
#pragma unroll
        for (int r = 1; r < R; ++r) {
            float2 w = __ldg(&tw[r * k * tstride]);
            if (sign > 0.0f) w.y = -w.y;
            v[r] = cmul(v[r], w);
        }
        dft_radix(v, R, sign);
        const int idx = jq * Ns * R + k;
        float2* dst = b + line * ls;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[(idx + r * Ns) * es] = v[r];
    }
    __syncthreads();
}

// Radices in the order 4,...,4, 2, 3,...,3, 5,...,5 (n = 2^a 3^b 5^c).
template <int NT>
__device__ float2* fft_lines(float2* a, float2* b, int n, int nlines, int ls, int es, const float2* __restrict__ tw,
                             float sign, bool line_fastest) {
    int Ns = 1, m = n;
    const FastDiv dl(nlines);
    while (m > 1) {
        int R;
        if (m % 4 == 0) { R = 4; fft_stage<4, NT>(a, b, n, nlines, ls, es, tw, sign, line_fastest, Ns, dl); }
        else if (m % 2 == 0) { R = 2; fft_stage<2, NT>(a, b, n, nlines, ls, es, tw, sign, line_fastest, Ns, dl); }
        else if (m % 3 == 0) { R = 3; fft_stage<3, NT>(a, b, n, nlines, ls, es, tw, sign, line_fastest, Ns, dl); }
        else { R = 5; fft_stage<5, NT>(a, b, n, nlines, ls, es, tw, sign, line_fastest, Ns, dl); }
        float2* t = a; a = b; b = t;
        Ns *= R;
        m /= R;
    }
    return a;
}

