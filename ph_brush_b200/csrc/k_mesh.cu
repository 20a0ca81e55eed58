// SPME mesh kernels: deterministic charge spreading, batched 3-D FFT passes
// (x/y planes resident in shared memory, z pencils in shared memory with the
// influence-function multiply fused between the forward and inverse z passes),
// potential-mesh readout.  Replaces k_spread_cubic + cuFFT R2C +
// k_recip_energy_and_apply of the reference (MC/src/pme.cu:140-249,384-422).
#include <cmath>
#include <cstring>
#include <string>
#include "common.cuh"
#include "engine.h"

// ---------------------------------------------------------------------------
// Mixed-radix Stockham autosort FFT over `nlines` lines held in shared memory
// (Govindaraju et al., "High performance discrete Fourier transforms on
// graphics processors", SC'08).  Element e of line l lives at l*ls + e*es.
// Returns the buffer that holds the result (a or b).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by sign*i
__device__ __forceinline__ float2 cmul_si(float2 a, float sign) { return make_float2(-sign * a.y, sign * a.x); }

__device__ __forceinline__ void dft_radix(float2* v, int R, float sign) {
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

template <int NT>
__device__ float2* fft_lines(float2* a, float2* b, int n, int nlines, int ls, int es, const float2* __restrict__ tw,
                             float sign, bool line_fastest) {
    int rad[16];
    const int ns = fft_plan(n, rad);
    int Ns = 1;
    for (int s = 0; s < ns; ++s) {
        const int R = rad[s];
        const int nb = n / R;
        const int tstride = n / (Ns * R);
        const int total = nb * nlines;
        for (int t = threadIdx.x; t < total; t += NT) {
            int line, j;
            if (line_fastest) { line = t % nlines; j = t / nlines; }
            else { j = t % nb; line = t / nb; }
            const int k = j % Ns;
            float2 v[5];
            const float2* src = a + line * ls;
#pragma unroll 5
            for (int r = 0; r < 5; ++r)
                if (r < R) v[r] = src[(j + r * nb) * es];
            for (int r = 1; r < R; ++r) {
                float2 w = __ldg(&tw[r * k * tstride]);
                if (sign > 0.0f) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
            dft_radix(v, R, sign);
            const int idx = (j / Ns) * Ns * R + k;
            float2* dst = b + line * ls;
            for (int r = 0; r < R; ++r) dst[(idx + r * Ns) * es] = v[r];
        }
        __syncthreads();
        float2* t = a; a = b; b = t;
        Ns *= R;
    }
    return a;
}

// ---------------------------------------------------------------------------
// Spreading: thread per slot; fixed-point (2^40) 64-bit atomics make the mesh
// bit-reproducible (integer addition is associative).
// ---------------------------------------------------------------------------
template <int P>
__global__ void k_spread(DevPtrs d, const int* __restrict__ rep_of, int total_slots, const int* __restrict__ dirty) {
    const int gs = blockIdx.x * blockDim.x + threadIdx.x;
    if (gs >= total_slots) return;
    const int r = rep_of[gs];
    if (dirty && !dirty[r]) return;
    if (d.flags[gs] & PHMC_F_GHOST) return;
    const float4 pq = d.posq[gs];
    if (pq.w == 0.0f) return;
    const RepDesc& D = d.desc[r];
    const int nx = D.mesh[0], ny = D.mesh[1], nz = D.mesh[2];
    float w[3][P];
    int base[3];
    const float g[3] = {pq.x / D.L[0] * (float)nx, pq.y / D.L[1] * (float)ny, pq.z / D.L[2] * (float)nz};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float fl = floorf(g[k]);
        bspline_weights<P>(g[k] - fl, w[k]);
        base[k] = (int)fl + P / 2 - P + 1;
    }
    unsigned long long* q = d.qfix + D.mesh_off;
    for (int c = 0; c < P; ++c) {
        const int zc = wrap_idx(base[2] + c, nz);
        for (int b = 0; b < P; ++b) {
            const int yb = wrap_idx(base[1] + b, ny);
            const float wyz = pq.w * w[1][b] * w[2][c];
            for (int a = 0; a < P; ++a) {
                const int xa = wrap_idx(base[0] + a, nx);
                const long long v = __double2ll_rn((double)(wyz * w[0][a]) * PHMC_FIX_SCALE);
                atomicAdd(q + ((size_t)zc * ny + yb) * nx + xa, (unsigned long long)v);
            }
        }
    }
}

// Place a unit charge exactly on mesh point 0 of every replica (to obtain the
// influence kernel G as the potential of that charge).
__global__ void k_unit_charge(DevPtrs d, int R) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    d.qfix[d.desc[r].mesh_off] = (unsigned long long)(long long)PHMC_FIX_SCALE;
}

// ---------------------------------------------------------------------------
// xy plane pass.  job = (replica, z).  forward: fixed-point charges -> complex
// spectrum along x then y (the fixed-point plane is cleared for the next
// spread).  inverse: complex -> real potential, y then x.
// ---------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(NT) k_plane(DevPtrs d, const int2* __restrict__ jobs, int forward, const int* __restrict__ dirty) {
    extern __shared__ float2 sm[];
    const int2 job = jobs[blockIdx.x];
    const int r = job.x, z = job.y;
    if (dirty && !dirty[r]) return;
    const RepDesc& D = d.desc[r];
    const int nx = D.mesh[0], ny = D.mesh[1];
    const int P = nx * ny;
    float2* a = sm;
    float2* b = sm + P;
    const size_t off = (size_t)D.mesh_off + (size_t)z * P;
    if (forward) {
        unsigned long long* q = d.qfix + off;
        for (int i = threadIdx.x; i < P; i += NT) {
            const long long v = (long long)q[i];
            q[i] = 0ull;
            a[i] = make_float2((float)((double)v * PHMC_FIX_INV), 0.0f);
        }
        __syncthreads();
        float2* res = fft_lines<NT>(a, b, nx, ny, nx, 1, d.twiddle + D.tw_off[0], -1.0f, false);
        float2* oth = (res == a) ? b : a;
        res = fft_lines<NT>(res, oth, ny, nx, 1, nx, d.twiddle + D.tw_off[1], -1.0f, true);
        float2* c = d.cmesh + off;
        for (int i = threadIdx.x; i < P; i += NT) c[i] = res[i];
    } else {
        const float2* c = d.cmesh + off;
        for (int i = threadIdx.x; i < P; i += NT) a[i] = c[i];
        __syncthreads();
        float2* res = fft_lines<NT>(a, b, ny, nx, 1, nx, d.twiddle + D.tw_off[1], 1.0f, true);
        float2* oth = (res == a) ? b : a;
        res = fft_lines<NT>(res, oth, nx, ny, nx, 1, d.twiddle + D.tw_off[0], 1.0f, false);
        float* phi = d.phi + off;
        for (int i = threadIdx.x; i < P; i += NT) phi[i] = res[i].x;
    }
}

// ---------------------------------------------------------------------------
// z pencil pass with the influence multiply fused: forward FFT along z,
// E += w(kx) * theta(k) |F(k)|^2, F *= theta, inverse FFT along z.
// job = (replica, y, x0); TX columns per job.
// theta(k) = elf * exp(-(pi/alpha)^2 m^2) / (pi V m^2 Bx By Bz)   (MC/src/pme.cu:212-223)
// ---------------------------------------------------------------------------
template <int NT, int TX>
__global__ void __launch_bounds__(NT) k_zpass(DevPtrs d, const int4* __restrict__ jobs, double* __restrict__ epart,
                                              const int* __restrict__ dirty) {
    extern __shared__ float2 sm[];
    __shared__ double red[40];
    const int4 job = jobs[blockIdx.x];
    const int r = job.x, y = job.y, x0 = job.z;
    if (dirty && !dirty[r]) { if (threadIdx.x == 0) epart[blockIdx.x] = 0.0; return; }
    const RepDesc& D = d.desc[r];
    const int nx = D.mesh[0], ny = D.mesh[1], nz = D.mesh[2];
    const int tx_n = min(TX, nx - x0);
    float2* a = sm;
    float2* b = sm + TX * nz;
    float2* c = d.cmesh + D.mesh_off;
    for (int e = threadIdx.x; e < nz * TX; e += NT) {
        const int z = e / TX, tx = e % TX;
        a[e] = (tx < tx_n) ? c[((size_t)z * ny + y) * nx + x0 + tx] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2* res = fft_lines<NT>(a, b, nz, TX, 1, TX, d.twiddle + D.tw_off[2], -1.0f, true);
    const float* mx = d.moduli + D.mod_off[0];
    const float* my = d.moduli + D.mod_off[1];
    const float* mz = d.moduli + D.mod_off[2];
    const int myi = (y <= ny / 2) ? y : y - ny;
    const float kyv = (float)myi / D.L[1];
    const float pv = 3.14159265358979323846f * (float)D.V;
    double e_loc = 0.0;
    for (int e = threadIdx.x; e < nz * TX; e += NT) {
        const int kz = e / TX, tx = e % TX;
        const int kx = x0 + tx;
        float2 F = res[e];
        float th = 0.0f;
        if (tx < tx_n && !(kx == 0 && y == 0 && kz == 0)) {
            const int mxi = (kx <= nx / 2) ? kx : kx - nx;
            const int mzi = (kz <= nz / 2) ? kz : kz - nz;
            const float kxv = (float)mxi / D.L[0], kzv = (float)mzi / D.L[2];
            const float m2 = kxv * kxv + kyv * kyv + kzv * kzv;
            const float den = m2 * pv * mx[kx] * my[y] * mz[kz];
            if (den > 0.0f) th = D.elf * expf(-D.ewald_factor * m2) / den;
            float wgt = 1.0f;
            if (D.ref_corner) wgt = (kx > nx / 2) ? 0.0f : ((kx == 0 || kx == nx / 2) ? 1.0f : 2.0f);
            e_loc += (double)(wgt * th) * ((double)F.x * F.x + (double)F.y * F.y);
        }
        res[e] = make_float2(F.x * th, F.y * th);
    }
    __syncthreads();
    float2* oth = (res == a) ? b : a;
    res = fft_lines<NT>(res, oth, nz, TX, 1, TX, d.twiddle + D.tw_off[2], 1.0f, true);
    for (int e = threadIdx.x; e < nz * TX; e += NT) {
        const int z = e / TX, tx = e % TX;
        if (tx < tx_n) c[((size_t)z * ny + y) * nx + x0 + tx] = res[e];
    }
    const double s = block_sum<NT>(e_loc, red);
    if (threadIdx.x == 0) epart[blockIdx.x] = 0.5 * s;
}

// Per-replica reduction of the z-pass energy partials (fixed order) and the
// energy bookkeeping of a potential-mesh rebuild.  mode 0: rebuild after MC
// (update tracked energies, record drift); mode 1: plain recompute (set E_rec).
__global__ void k_flush_reduce(DevPtrs d, const int* __restrict__ zjob_off, const double* __restrict__ epart, int R,
                               int mode, const int* __restrict__ dirty) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    if (dirty && !dirty[r]) return;
    double s = 0.0;
    for (int k = zjob_off[r]; k < zjob_off[r + 1]; ++k) s += epart[k];
    RepState& S = d.state[r];
    S.E_rec_flush = s;
    if (mode == 0) {
        S.drift = fabs(S.E_rec - s);
        S.E += s - S.E_rec;
        S.E_rec = s;
        S.flushes += 1;
        d.dirty[r] = 0;
    } else {
        S.E_rec = s;
    }
}

// Copy the non-negative octant of the potential of a unit charge (the
// influence kernel G, even in each axis) into the compact G table.
__global__ void k_extract_octant(DevPtrs d, int r) {
    const RepDesc& D = d.desc[r];
    const int ox = D.oct[0], oy = D.oct[1], oz = D.oct[2];
    const int total = ox * oy * oz;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int x = i % ox, y = (i / ox) % oy, z = i / (ox * oy);
        d.goct[D.oct_off + i] = d.phi[D.mesh_off + ((size_t)z * D.mesh[1] + y) * D.mesh[0] + x];
    }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
void launch_spread(Engine& E, const int* dirty, cudaStream_t st) {
    const int nt = 256, nb = (E.total_slots + nt - 1) / nt;
    switch (E.order) {
        case 4: k_spread<4><<<nb, nt, 0, st>>>(E.d, E.d_rep_of, E.total_slots, dirty); break;
        case 5: k_spread<5><<<nb, nt, 0, st>>>(E.d, E.d_rep_of, E.total_slots, dirty); break;
        case 6: k_spread<6><<<nb, nt, 0, st>>>(E.d, E.d_rep_of, E.total_slots, dirty); break;
    }
}

void launch_fft_pipeline(Engine& E, const int* dirty, int mode, cudaStream_t st) {
    k_plane<256><<<E.n_plane_jobs, 256, E.plane_smem, st>>>(E.d, E.d_plane_jobs, 1, dirty);
    k_zpass<256, ZPASS_TX><<<E.n_zjobs, 256, E.zpass_smem, st>>>(E.d, E.d_zjobs, E.d_epart, dirty);
    k_plane<256><<<E.n_plane_jobs, 256, E.plane_smem, st>>>(E.d, E.d_plane_jobs, 0, dirty);
    k_flush_reduce<<<(E.R + 127) / 128, 128, 0, st>>>(E.d, E.d_zjob_off, E.d_epart, E.R, mode, dirty);
}

void launch_unit_charge(Engine& E, cudaStream_t st) { k_unit_charge<<<(E.R + 127) / 128, 128, 0, st>>>(E.d, E.R); }

void launch_extract_octant(Engine& E, int r, cudaStream_t st) { k_extract_octant<<<148, 256, 0, st>>>(E.d, r); }

// The cap is the device's opt-in maximum (not this engine's need), so that
// engines with different meshes can coexist on one device.
template <typename K>
static cudaError_t raise_dynamic_smem_cap(K kernel, int device, size_t need) {
    int optin = 0;
    cudaError_t e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, kernel);
    if (e != cudaSuccess) return e;
    const int cap = optin - (int)fa.sharedSizeBytes;  // static shared memory counts against the opt-in limit
    if (cap < (int)need) return cudaErrorInvalidValue;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, cap);
}

cudaError_t mesh_set_smem_limits(Engine& E) {
    cudaError_t e = raise_dynamic_smem_cap(k_plane<256>, E.device, E.plane_smem);
    if (e != cudaSuccess) return e;
    return raise_dynamic_smem_cap(k_zpass<256, ZPASS_TX>, E.device, E.zpass_smem);
}
