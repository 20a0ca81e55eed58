// Potential-mesh rebuild for meshes with even nx: three passes over the
// half-spectrum mesh of each replica's fixed-point charge mesh.
//
//  The charge mesh Q (2^40 fixed point, 64-bit integers: deterministic, order-
//  independent sums) covers the planes of each replica's wall band.  It is kept
//  current incrementally: the MC kernel adds the stencil values of every accepted
//  change (old charges out, new charges in) with integer atomics, computed with the
//  same exactly-rounded weights as the full spread (k_band_spread, run at every full
//  recompute), so Q always equals a fresh spread of the current configuration.
//
//  k_band_spread (replica, z): gather the charges whose order-P stencils reach plane
//            z from the cell list, accumulate them in a shared-memory fixed-point
//            plane, store it to Q.
//  k_rb_fwd  (replica, z): Q plane -> float, real-to-complex FFT along x (length
//            nx/2 complex FFT of packed pairs + split) and complex FFT along y;
//            writes (nx/2+1) x ny complex values.
//  k_rb_zpass / k_rb_zreg (column tiles): FFT along z, E += w theta |F|^2,
//            F *= theta, inverse FFT along z.
//  k_rb_inv  (replica, z): inverse FFT along y, complex-to-real along x; writes
//            the real potential plane.
// With hard walls the charges stay in a band of planes (RepDesc::zb_lo, zb_n) and the
// MC kernel reads the potential only there: the first and last passes run on the
// band's planes, the z pass loads and stores only those (the rest of the input is
// zero).  The unit-charge rebuild of the influence kernel computes every plane.
// Replaces the memset + k_spread_cubic + cuFFT R2C + influence kernel chain of
// the reference (MC/src/pme.cu:140-249,362,384-422).
#include <algorithm>
#include "common.cuh"
#include "engine.h"
#include "fft.cuh"
#include "fft_reg.cuh"

template <int P, int NT>
__global__ void __launch_bounds__(NT) k_band_spread(DevPtrs d, const int2* __restrict__ jobs) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    const int2 job = jobs[blockIdx.x];
    const int r = job.x, z = job.y;
    const RepDesc& D = d.desc[r];
    const int nx = D.mesh[0], ny = D.mesh[1], nz = D.mesh[2];
    unsigned long long* qp = reinterpret_cast<unsigned long long*>(sm_raw);
    int* s_cnt = reinterpret_cast<int*>(qp + nx * ny);
    const int tid = threadIdx.x;
    for (int i = tid; i < nx * ny; i += NT) qp[i] = 0ull;
    __syncthreads();
    // floor(g_z) of a contributing charge lies in [z - P/2, z - P/2 + P - 1] (mod nz)
    const float hz = D.L[2] / (float)nz;
    const float lo = (float)(z - P / 2) * hz, hi = (float)(z - P / 2 + P) * hz;
    const int ncz = D.ncell[2], ncxy = D.ncell[0] * D.ncell[1];
    // the cell layers of [lo, hi), widened by a rounding margin (the exact test is per charge)
    int c_lo = (int)floorf((lo - 1e-3f * hz) * D.cell_scale[2]), c_hi = (int)floorf((hi + 1e-3f * hz) * D.cell_scale[2]);
    int nlay = c_hi - c_lo + 1;
    if (nlay > ncz) { nlay = ncz; c_lo = 0; }
    const int ncell = nlay * ncxy;
    // member counts of every cell in the layers, then an exclusive scan, so that the
    // (cell, member) items spread over all threads with independent loads
    __shared__ int s_wsum[NT / 32 + 1];
    // cell of item cc: layer cc / ncxy (wrapped in z), in-layer index cc % ncxy
    auto cell_of_item = [&](int cc) {
        const int lay = cc / ncxy, cxy = cc - lay * ncxy;
        int cz = (c_lo + lay) % ncz;
        cz += (cz < 0) ? ncz : 0;
        return cz * ncxy + cxy;
    };
    for (int cc = tid; cc < ncell; cc += NT)
        s_cnt[cc] = min(d.cell_count[D.cell_off + cell_of_item(cc)], D.cell_cap);
    __syncthreads();
    {   // block scan: each thread a contiguous chunk, then the chunk totals
        const int per = (ncell + NT - 1) / NT;
        const int b0 = min(ncell, tid * per), b1 = min(ncell, b0 + per);
        int sum = 0;
        for (int i = b0; i < b1; ++i) sum += s_cnt[i];
        int x = sum;
        const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s_wsum[warp] = x;
        __syncthreads();
        if (tid == 0) {
            int acc = 0;
            for (int w = 0; w < NT / 32; ++w) { const int v = s_wsum[w]; s_wsum[w] = acc; acc += v; }
            s_wsum[NT / 32] = acc;
        }
        __syncthreads();
        int run = s_wsum[warp] + x - sum;
        for (int i = b0; i < b1; ++i) { const int v = s_cnt[i]; s_cnt[i] = run; run += v; }
        if (tid == NT - 1) s_cnt[ncell] = s_wsum[NT / 32];
    }
    __syncthreads();
    const int total = s_cnt[ncell];
    for (int it = tid; it < total; it += NT) {
        int lo2 = 0, hi2 = ncell - 1;  // last cell whose offset <= it
        while (lo2 < hi2) {
            const int mid = (lo2 + hi2 + 1) >> 1;
            if (s_cnt[mid] <= it) lo2 = mid; else hi2 = mid - 1;
        }
        const int c = cell_of_item(lo2);
        const int k = it - s_cnt[lo2];
        const float4 pq = d.posq[D.slot_off + d.cell_list[((size_t)D.cell_off + c) * D.cell_cap + k]];
        if (pq.w == 0.0f) continue;
        float w[3][P];
        int base[3];
        qmesh_stencil<P>(D, pq, w, base);
        int ci = z - base[2];
        ci %= nz;
        ci += (ci < 0) ? nz : 0;
        if (ci >= P) continue;
        float wz = 0.0f;  // select: w[2][ci] without a dynamic index
#pragma unroll
        for (int j = 0; j < P; ++j) wz = (j == ci) ? w[2][j] : wz;
#pragma unroll
        for (int bb = 0; bb < P; ++bb) {
            int yb = base[1] + bb;
            yb += (yb < 0) ? ny : 0;
            yb -= (yb >= ny) ? ny : 0;
#pragma unroll
            for (int aa = 0; aa < P; ++aa) {
                int xa = base[0] + aa;
                xa += (xa < 0) ? nx : 0;
                xa -= (xa >= nx) ? nx : 0;
                atomicAdd(&qp[yb * nx + xa], (unsigned long long)qmesh_value(pq.w, w[0][aa], w[1][bb], wz));
            }
        }
    }
    __syncthreads();
    int zrel = z - D.zb_lo;
    zrel += (zrel < 0) ? nz : 0;
    unsigned long long* q = d.qband + D.qb_off + (size_t)zrel * nx * ny;
    for (int i = tid; i < nx * ny; i += NT) q[i] = qp[i];
}

template <int NT>
__global__ void __launch_bounds__(NT) k_rb_fwd(DevPtrs d, const int2* __restrict__ jobs, int unit_charge,
                                               const int* __restrict__ dirty) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    const int2 job = jobs[blockIdx.x];
    const int r = job.x, z = job.y;
    if (dirty && !dirty[r]) return;
    const RepDesc& D = d.desc[r];
    const int nx = D.mesh[0], ny = D.mesh[1], nz = D.mesh[2];
    const int M = nx / 2, nxh = M + 1;
    // two complex buffers of nxh x ny; the real plane Q[y][x] (row length nx) is loaded as
    // the packed pairs a[y*M + j] = (Q[y][2j], Q[y][2j+1])
    float2* a = reinterpret_cast<float2*>(sm_raw);
    float2* b = a + nxh * ny;
    const int tid = threadIdx.x;
    if (unit_charge) {  // a unit charge on mesh point 0 (the influence kernel's source)
        for (int i = tid; i < M * ny; i += NT) a[i] = make_float2((z == 0 && i == 0) ? 1.0f : 0.0f, 0.0f);
    } else {
        int zrel = z - D.zb_lo;
        zrel += (zrel < 0) ? nz : 0;
        const ulonglong2* q = reinterpret_cast<const ulonglong2*>(d.qband + D.qb_off + (size_t)zrel * nx * ny);
        for (int i = tid; i < M * ny; i += NT) {
            const ulonglong2 v = q[i];
            a[i] = make_float2((float)((double)(long long)v.x * PHMC_FIX_INV), (float)((double)(long long)v.y * PHMC_FIX_INV));
        }
    }
    __syncthreads();
    float2* zr = fft_lines<NT>(a, b, M, ny, M, 1, d.twiddle + D.tw_off_h, -1.0f, false);
    float2* xo = (zr == a) ? b : a;
    const float2* twn = d.twiddle + D.tw_off[0];  // exp(-2 pi i k / nx)
    // split: X_k = 1/2 (Z_k + conj Z_{M-k}) - i/2 W^k (Z_k - conj Z_{M-k}), k = 0..M
    for (int i = tid; i < nxh * ny; i += NT) {
        const int y = i / nxh, k = i - y * nxh;
        const float2 zk = zr[y * M + (k == M ? 0 : k)];
        float2 zc = zr[y * M + (k == 0 ? 0 : M - k)];
        zc.y = -zc.y;
        const float2 w = twn[k];
        const float2 s = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y + zc.y));
        const float2 df = make_float2(0.5f * (zk.x - zc.x), 0.5f * (zk.y - zc.y));
        const float2 wd = cmul(w, df);  // W * (Z_k - conj Z_{M-k}) / 2
        xo[y * nxh + k] = make_float2(s.x + wd.y, s.y - wd.x);  // s - i * wd
    }
    __syncthreads();
    float2* res = fft_lines<NT>(xo, zr, ny, nxh, 1, nxh, d.twiddle + D.tw_off[1], -1.0f, true);
    float2* c = d.cmesh + D.meshh_off + (size_t)z * ny * nxh;
    for (int i = tid; i < nxh * ny; i += NT) c[i] = res[i];
}

// z pencils of the half spectrum; job = (replica, y, x0, width <= ZPASS_TX).
template <int NT, int TX>
__global__ void __launch_bounds__(NT) k_rb_zpass(DevPtrs d, const int4* __restrict__ jobs, double* __restrict__ epart,
                                                 const int* __restrict__ dirty, int full) {
    extern __shared__ float2 sm[];
    __shared__ double red[40];
    const int4 job = jobs[blockIdx.x];
    const int r = job.x, y = job.y, x0 = job.z, tw_n = job.w;
    if (dirty && !dirty[r]) { if (threadIdx.x == 0) epart[blockIdx.x] = 0.0; return; }
    const RepDesc& D = d.desc[r];
    const int nx = D.mesh[0], ny = D.mesh[1], nz = D.mesh[2];
    const int M = nx / 2, nxh = M + 1;
    float2* a = sm;
    float2* b = sm + TX * nz;
    float2* c = d.cmesh + D.meshh_off;
    const int zlo = full ? 0 : D.zb_lo, zbn = full ? nz : D.zb_n;
    auto in_band = [&](int z) { int t = z - zlo; t += (t < 0) ? nz : 0; return t < zbn; };
    for (int e = threadIdx.x; e < nz * TX; e += NT) {
        const int z = e / TX, tx = e - z * TX;
        a[e] = (tx < tw_n && in_band(z)) ? c[((size_t)z * ny + y) * nxh + x0 + tx] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2* res = fft_lines<NT>(a, b, nz, TX, 1, TX, d.twiddle + D.tw_off[2], -1.0f, true);
    const float2* thx = d.thtab + D.th_off[0];
    const float2 fy = d.thtab[D.th_off[1] + y];
    const float2* thz = d.thtab + D.th_off[2];
    double e_loc = 0.0;
    for (int e = threadIdx.x; e < nz * TX; e += NT) {
        const int kz = e / TX, tx = e - kz * TX;
        const int kx = x0 + tx;
        const float2 F = res[e];
        float th = 0.0f;
        if (tx < tw_n && !(kx == 0 && y == 0 && kz == 0)) {
            // theta = th_c tx ty tz / |k|^2 from the per-axis factor tables
            const float2 fx = __ldg(&thx[kx]), fz = __ldg(&thz[kz]);
            th = __fdividef(D.th_c * fx.x * fy.x * fz.x, fx.y + fy.y + fz.y);
            const float wgt = (kx == 0 || kx == M) ? 1.0f : 2.0f;  // half spectrum, Hermitian partners counted
            e_loc += (double)(wgt * th) * ((double)F.x * F.x + (double)F.y * F.y);
        }
        res[e] = make_float2(F.x * th, F.y * th);
    }
    __syncthreads();
    float2* oth = (res == a) ? b : a;
    res = fft_lines<NT>(res, oth, nz, TX, 1, TX, d.twiddle + D.tw_off[2], 1.0f, true);
    for (int e = threadIdx.x; e < nz * TX; e += NT) {
        const int z = e / TX, tx = e - z * TX;
        if (tx < tw_n && in_band(z)) c[((size_t)z * ny + y) * nxh + x0 + tx] = res[e];
    }
    const double s = block_sum<NT>(e_loc, red);
    if (threadIdx.x == 0) epart[blockIdx.x] = 0.5 * s;
}

// z pencils with register-resident DFTs, nz = N1 * N2: TX consecutive columns of the
// flattened half-spectrum plane (ny x (nx/2+1)); job = (replica, first column, columns, 0).
//   stage A: per (n2, column) the length-N1 DFT over x[N2 n1 + n2] straight from global
//            memory, times W_nz^(n2 k1), into shared memory at [k1][n2];
//   stage B: per (k1, column) the length-N2 DFT over n2 gives F(kz = k1 + N1 k2);
//            E += w theta |F|^2, F *= theta; the inverse length-N2 DFT and W_nz^(-n2 k1)
//            go back to the same shared-memory row;
//   stage A': per (n2, column) the inverse length-N1 DFT over k1, stored to global memory.
// Shared memory is touched twice per direction instead of once per radix stage.
template <int N1, int N2, int NT, int TX>
__global__ void __launch_bounds__(NT) k_rb_zreg(DevPtrs d, const int4* __restrict__ jobs, double* __restrict__ epart,
                                                const int* __restrict__ dirty, int full) {
    constexpr int N = N1 * N2;
    static_assert((TX & (TX - 1)) == 0, "TX must be a power of two");
    extern __shared__ float2 sm[];
    __shared__ double red[40];
    const int4 job = jobs[blockIdx.x];
    const int r = job.x, c0 = job.y, ncol = job.z;
    if (dirty && !dirty[r]) { if (threadIdx.x == 0) epart[blockIdx.x] = 0.0; return; }
    const RepDesc& D = d.desc[r];
    const int nx = D.mesh[0], ny = D.mesh[1];
    const int M = nx / 2, nxh = M + 1;
    const size_t plane = (size_t)ny * nxh;
    float2* s = sm;            // [k1][n2][column]
    float2* tw = sm + N * TX;  // exp(-2 pi i j / nz)
    float2* thz = tw + N;      // z influence factor and k_z^2 per kz
    float2* c = d.cmesh + D.meshh_off + c0;
    // planes outside the wall band hold no charge (zero input) and are not read back
    const int zlo = full ? 0 : D.zb_lo, zbn = full ? N : D.zb_n;
    auto in_band = [&](int z) { int t = z - zlo; t += (t < 0) ? N : 0; return t < zbn; };
    for (int i = threadIdx.x; i < N; i += NT) { tw[i] = d.twiddle[D.tw_off[2] + i]; thz[i] = d.thtab[D.th_off[2] + i]; }
    // stage A: the loads of the first round go out before the barrier that publishes tw
    for (int base = 0; base < N2 * TX; base += NT) {
        const int it = base + threadIdx.x;
        const int n2 = it / TX, col = it & (TX - 1);
        const bool act = it < N2 * TX;
        float2 v[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1)
            v[n1] = (act && col < ncol && in_band(N2 * n1 + n2)) ? c[(size_t)(N2 * n1 + n2) * plane + col]
                                                                 : make_float2(0.f, 0.f);
        if (base == 0) __syncthreads();
        if (act) {
            rfft::rdft<N1, -1>(v);
            s[n2 * TX + col] = v[0];
#pragma unroll
            for (int k1 = 1; k1 < N1; ++k1) s[(k1 * N2 + n2) * TX + col] = cmul(v[k1], tw[n2 * k1]);
        }
    }
    __syncthreads();
    double e_loc = 0.0;
    for (int it = threadIdx.x; it < N1 * TX; it += NT) {
        const int k1 = it / TX, col = it & (TX - 1);
        float2 u[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) u[n2] = s[(k1 * N2 + n2) * TX + col];
        rfft::rdft<N2, -1>(u);
        const int idx = c0 + col;
        const int y = idx / nxh, kx = idx - y * nxh;
        const bool valid = col < ncol;
        // theta = th_c tx ty tz / |k|^2 from the per-axis factor tables (column part once)
        const float2 fx = valid ? d.thtab[D.th_off[0] + kx] : make_float2(0.0f, 1.0f);
        const float2 fy = valid ? d.thtab[D.th_off[1] + y] : make_float2(0.0f, 1.0f);
        const float cxy = D.th_c * fx.x * fy.x, kxy2 = fx.y + fy.y;
        const float wgt = (kx == 0 || kx == M) ? 1.0f : 2.0f;  // half spectrum, Hermitian partners counted
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) {
            const int kz = k1 + N1 * k2;
            const float2 F = u[k2];
            float th = 0.0f;
            if (valid && !(kx == 0 && y == 0 && kz == 0)) {
                const float2 fz = thz[kz];
                th = __fdividef(cxy * fz.x, kxy2 + fz.y);
                e_loc += (double)(wgt * th) * ((double)F.x * F.x + (double)F.y * F.y);
            }
            u[k2] = make_float2(F.x * th, F.y * th);
        }
        rfft::rdft<N2, 1>(u);
        s[k1 * N2 * TX + col] = u[0];
#pragma unroll
        for (int n2 = 1; n2 < N2; ++n2) {
            float2 w = tw[n2 * k1];
            w.y = -w.y;
            s[(k1 * N2 + n2) * TX + col] = cmul(u[n2], w);
        }
    }
    __syncthreads();
    for (int it = threadIdx.x; it < N2 * TX; it += NT) {
        const int n2 = it / TX, col = it & (TX - 1);
        float2 v[N1];
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) v[k1] = s[(k1 * N2 + n2) * TX + col];
        rfft::rdft<N1, 1>(v);
        if (col < ncol) {
#pragma unroll
            for (int n1 = 0; n1 < N1; ++n1)
                if (in_band(N2 * n1 + n2)) c[(size_t)(N2 * n1 + n2) * plane + col] = v[n1];
        }
    }
    const double es = block_sum<NT>(e_loc, red);
    if (threadIdx.x == 0) epart[blockIdx.x] = 0.5 * es;
}

// (id, nz, N1, N2) of the register z passes; id 0 = shared-memory z pass.  The first entry
// of an nz is its default; the others are the splits the autotuner also tries.
#define ZREG_LIST(X) X(1, 48, 8, 6) X(2, 128, 16, 8) X(3, 162, 18, 9) X(4, 192, 16, 12) X(5, 216, 24, 9) \
                     X(6, 243, 27, 9) X(7, 256, 16, 16) X(8, 288, 32, 9) X(9, 384, 32, 12)            \
                     X(10, 48, 6, 8) X(11, 128, 8, 16) X(12, 162, 9, 18) X(13, 192, 12, 16)           \
                     X(14, 216, 9, 24) X(15, 243, 9, 27) X(16, 288, 9, 32) X(17, 384, 24, 16)         \
                     X(18, 384, 12, 32)
constexpr int ZREG_NT(int n2) { return (n2 * ZREG_TX + 31) / 32 * 32 > 256 ? 256 : (n2 * ZREG_TX + 31) / 32 * 32; }

int zreg_variant(int nz) {
#define ZREG_CASE(id, n, a, b) if (nz == n) return id;
    ZREG_LIST(ZREG_CASE)
#undef ZREG_CASE
    return 0;
}
int zreg_variants(int nz, int* ids, int max_ids) {
    int n = 0;
#define ZREG_ALL(id, nn, a, b) if (nz == nn && n < max_ids) ids[n++] = id;
    ZREG_LIST(ZREG_ALL)
#undef ZREG_ALL
    return n;
}
void zreg_split(int id, int* n1, int* n2) {
    *n1 = 0; *n2 = 0;
#define ZREG_SPLIT(i, nn, a, b) if (id == i) { *n1 = a; *n2 = b; }
    ZREG_LIST(ZREG_SPLIT)
#undef ZREG_SPLIT
}
size_t zreg_smem(int nz) { return (size_t)(ZREG_TX + 2) * nz * sizeof(float2); }

template <int NT>
__global__ void __launch_bounds__(NT) k_rb_inv(DevPtrs d, const int2* __restrict__ jobs, const int* __restrict__ dirty) {
    extern __shared__ float2 sm[];
    const int2 job = jobs[blockIdx.x];
    const int r = job.x, z = job.y;
    if (dirty && !dirty[r]) return;
    const RepDesc& D = d.desc[r];
    const int nx = D.mesh[0], ny = D.mesh[1];
    const int M = nx / 2, nxh = M + 1;
    float2* a = sm;
    float2* b = sm + nxh * ny;
    const float2* c = d.cmesh + D.meshh_off + (size_t)z * ny * nxh;
    for (int i = threadIdx.x; i < nxh * ny; i += NT) a[i] = c[i];
    __syncthreads();
    float2* xr = fft_lines<NT>(a, b, ny, nxh, 1, nxh, d.twiddle + D.tw_off[1], 1.0f, true);
    float2* zo = (xr == a) ? b : a;
    const float2* twn = d.twiddle + D.tw_off[0];
    // merge: Z'_k = (X_k + conj X_{M-k}) + i W^{-k} (X_k - conj X_{M-k}), k = 0..M-1
    for (int i = threadIdx.x; i < M * ny; i += NT) {
        const int y = i / M, k = i - y * M;
        const float2 A = xr[y * nxh + k];
        float2 B = xr[y * nxh + (M - k)];
        B.y = -B.y;
        float2 w = twn[k];
        w.y = -w.y;  // W^{-k}
        const float2 s = make_float2(A.x + B.x, A.y + B.y);
        const float2 wd = cmul(w, make_float2(A.x - B.x, A.y - B.y));
        zo[y * M + k] = make_float2(s.x - wd.y, s.y + wd.x);  // s + i * wd
    }
    __syncthreads();
    float2* zz = fft_lines<NT>(zo, xr, M, ny, M, 1, d.twiddle + D.tw_off_h, 1.0f, false);
    float* phi = d.phi + D.mesh_off + (size_t)z * ny * nx;
    for (int i = threadIdx.x; i < M * ny; i += NT) {
        const int y = i / M, j = i - y * M;
        phi[y * nx + 2 * j] = zz[i].x;
        phi[y * nx + 2 * j + 1] = zz[i].y;
    }
}

// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// First and last passes with register-resident DFTs, for square lateral meshes
// n = nx = ny in the PLANE_LIST set (one block per (replica, z) plane, the
// replica's n picked at run time).  x: one thread per row, the row's n/2 packed
// complex values in registers (a row stride of odd length in float2 keeps the
// rows' shared-memory accesses free of bank conflicts); y: n = N1 * N2 in two
// register stages over the n/2 + 1 columns.  Shared memory is passed once per
// stage instead of once per radix stage.
// ---------------------------------------------------------------------------
#define PLANE_LIST(X) X(16, 4, 4) X(32, 8, 4) X(36, 6, 6) X(48, 8, 6) X(54, 9, 6) X(64, 8, 8)
constexpr int plane_ms(int m) { return (m % 2 == 0) ? m + 1 : m + 2; }  // odd row stride (float2)
constexpr int PLANE_NT = 128;
constexpr int PLANE_STAGE_BYTES = 64 * 64 * 8;  // one staged plane of the largest listed lateral mesh

// qs: the plane's fixed-point charges already staged in shared memory (the pipelined
// pass), or null to read them from global memory.
template <int N, int N1, int N2, int NT>
__device__ void plane_fwd(const DevPtrs& d, const RepDesc& D, int z, int unit_charge, float2* sa, float2* sb,
                          const ulonglong2* qs = nullptr) {
    constexpr int M = N / 2, NXH = M + 1, MS = plane_ms(M);
    static_assert(N1 * N2 == N, "y split");
    const int tid = threadIdx.x;
    float2* xa = sa;  // [y][j] packed real pairs, row stride MS; later the y stage-A output [k1 N2 + n2][k]
    float2* xb = sb;  // [y][k] after the split, row stride NXH
    if (unit_charge) {  // a unit charge on mesh point 0 (the influence kernel's source)
        for (int i = tid; i < N * M; i += NT) {
            const int y = i / M, j = i - y * M;
            xa[y * MS + j] = make_float2((z == 0 && i == 0) ? 1.0f : 0.0f, 0.0f);
        }
    } else {
        int zrel = z - D.zb_lo;
        zrel += (zrel < 0) ? D.mesh[2] : 0;
        const ulonglong2* q = qs ? qs : reinterpret_cast<const ulonglong2*>(d.qband + D.qb_off + (size_t)zrel * N * N);
        // batches of LB loads issued back to back before their shared-memory stores (the stores
        // could alias the loads as far as the compiler knows, so it would not hoist them)
        constexpr int LB = 8;
        for (int i0 = tid; i0 < N * M; i0 += LB * NT) {
            ulonglong2 v[LB];
#pragma unroll
            for (int u = 0; u < LB; ++u) {
                const int i = i0 + u * NT;
                if (i < N * M) v[u] = q[i];
            }
#pragma unroll
            for (int u = 0; u < LB; ++u) {
                const int i = i0 + u * NT;
                if (i >= N * M) break;
                const int y = i / M, j = i - y * M;
                xa[y * MS + j] = make_float2((float)((double)(long long)v[u].x * PHMC_FIX_INV),
                                             (float)((double)(long long)v[u].y * PHMC_FIX_INV));
            }
        }
    }
    __syncthreads();
    for (int y = tid; y < N; y += NT) {  // x: length-M DFT of the packed pairs of row y
        float2 v[M];
#pragma unroll
        for (int j = 0; j < M; ++j) v[j] = xa[y * MS + j];
        rfft::rdft<M, -1>(v);
#pragma unroll
        for (int j = 0; j < M; ++j) xa[y * MS + j] = v[j];
    }
    __syncthreads();
    const float2* twn = d.twiddle + D.tw_off[0];  // exp(-2 pi i k / nx)
    // split: X_k = 1/2 (Z_k + conj Z_{M-k}) - i/2 W^k (Z_k - conj Z_{M-k}), k = 0..M
    for (int i = tid; i < N * NXH; i += NT) {
        const int y = i / NXH, k = i - y * NXH;
        const float2 zk = xa[y * MS + (k == M ? 0 : k)];
        float2 zc = xa[y * MS + (k == 0 ? 0 : M - k)];
        zc.y = -zc.y;
        const float2 w = twn[k];
        const float2 s = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y + zc.y));
        const float2 df = make_float2(0.5f * (zk.x - zc.x), 0.5f * (zk.y - zc.y));
        const float2 wd = cmul(w, df);
        xb[y * NXH + k] = make_float2(s.x + wd.y, s.y - wd.x);
    }
    __syncthreads();
    const float2* twy = d.twiddle + D.tw_off[1];  // exp(-2 pi i j / ny)
    for (int it = tid; it < N2 * NXH; it += NT) {  // y stage A: DFT over n1 of rows N2 n1 + n2, times W^(n2 k1)
        const int n2 = it / NXH, k = it - n2 * NXH;
        float2 v[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) v[n1] = xb[(N2 * n1 + n2) * NXH + k];
        rfft::rdft<N1, -1>(v);
        xa[n2 * NXH + k] = v[0];
#pragma unroll
        for (int k1 = 1; k1 < N1; ++k1) xa[(k1 * N2 + n2) * NXH + k] = cmul(v[k1], twy[n2 * k1]);
    }
    __syncthreads();
    float2* c = d.cmesh + D.meshh_off + (size_t)z * N * NXH;
    for (int it = tid; it < N1 * NXH; it += NT) {  // y stage B: DFT over n2 gives row ky = k1 + N1 k2
        const int k1 = it / NXH, k = it - k1 * NXH;
        float2 u[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) u[n2] = xa[(k1 * N2 + n2) * NXH + k];
        rfft::rdft<N2, -1>(u);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) c[(k1 + N1 * k2) * NXH + k] = u[k2];
    }
}

template <int N, int N1, int N2, int NT>
__device__ void plane_inv(const DevPtrs& d, const RepDesc& D, int z, float2* sa, float2* sb) {
    constexpr int M = N / 2, NXH = M + 1, MS = plane_ms(M);
    const int tid = threadIdx.x;
    float2* xa = sa;
    float2* xb = sb;
    const float2* c = d.cmesh + D.meshh_off + (size_t)z * N * NXH;
    const float2* twy = d.twiddle + D.tw_off[1];
    for (int it = tid; it < N1 * NXH; it += NT) {  // inverse y stage B: over k2, then W^(-n2 k1)
        const int k1 = it / NXH, k = it - k1 * NXH;
        float2 u[N2];
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) u[k2] = c[(k1 + N1 * k2) * NXH + k];
        rfft::rdft<N2, 1>(u);
        xa[k1 * N2 * NXH + k] = u[0];
#pragma unroll
        for (int n2 = 1; n2 < N2; ++n2) {
            float2 w = twy[n2 * k1];
            w.y = -w.y;
            xa[(k1 * N2 + n2) * NXH + k] = cmul(u[n2], w);
        }
    }
    __syncthreads();
    for (int it = tid; it < N2 * NXH; it += NT) {  // inverse y stage A: over k1 gives row N2 n1 + n2
        const int n2 = it / NXH, k = it - n2 * NXH;
        float2 v[N1];
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) v[k1] = xa[(k1 * N2 + n2) * NXH + k];
        rfft::rdft<N1, 1>(v);
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) xb[(N2 * n1 + n2) * NXH + k] = v[n1];
    }
    __syncthreads();
    const float2* twn = d.twiddle + D.tw_off[0];
    // merge: Z'_k = (X_k + conj X_{M-k}) + i W^{-k} (X_k - conj X_{M-k}), k = 0..M-1
    for (int i = tid; i < N * M; i += NT) {
        const int y = i / M, k = i - y * M;
        const float2 A = xb[y * NXH + k];
        float2 B = xb[y * NXH + (M - k)];
        B.y = -B.y;
        float2 w = twn[k];
        w.y = -w.y;
        const float2 s = make_float2(A.x + B.x, A.y + B.y);
        const float2 wd = cmul(w, make_float2(A.x - B.x, A.y - B.y));
        xa[y * MS + k] = make_float2(s.x - wd.y, s.y + wd.x);
    }
    __syncthreads();
    for (int y = tid; y < N; y += NT) {  // inverse x: length-M DFT of row y's packed pairs
        float2 v[M];
#pragma unroll
        for (int j = 0; j < M; ++j) v[j] = xa[y * MS + j];
        rfft::rdft<M, 1>(v);
#pragma unroll
        for (int j = 0; j < M; ++j) xa[y * MS + j] = v[j];
    }
    __syncthreads();
    float2* phi = reinterpret_cast<float2*>(d.phi + D.mesh_off + (size_t)z * N * N);
    for (int i = tid; i < N * M; i += NT) {  // the real plane: row y, points 2j and 2j + 1
        const int y = i / M, j = i - y * M;
        phi[i] = xa[y * MS + j];
    }
}

template <int NT>
__global__ void __launch_bounds__(NT) k_rb_fwd_reg(DevPtrs d, const int2* __restrict__ jobs, int unit_charge,
                                                   const int* __restrict__ dirty) {
    extern __shared__ __align__(16) float2 psm[];
    const int2 job = jobs[blockIdx.x];
    const int r = job.x, z = job.y;
    if (dirty && !dirty[r]) return;
    const RepDesc& D = d.desc[r];
    const int n = D.mesh[0];
    float2* sa = psm;
    float2* sb = psm + n * plane_ms(n / 2);
    switch (n) {
#define PLANE_FWD(nn, a, b) case nn: plane_fwd<nn, a, b, NT>(d, D, z, unit_charge, sa, sb); break;
        PLANE_LIST(PLANE_FWD)
#undef PLANE_FWD
        default: break;
    }
}

// Pipelined first pass: persistent blocks walk the band-plane jobs with a stride of the
// grid; while a block transforms one plane, the next plane's fixed-point charges (N^2
// 8-byte values, contiguous) arrive in the other half of a two-stage shared-memory
// buffer by a bulk asynchronous copy (this GPU's own memory, no multicast), so the
// loads of the planes overlap the FFT work instead of opening every block.  Waits are
// bounded: a copy that does not arrive records PHMC_ERR_BUDGET in the replica's state
// and the block stops (the rebuild is then reported as failed).
template <int NT>
__global__ void __launch_bounds__(NT) k_rb_fwd_pipe(DevPtrs d, const int2* __restrict__ jobs, int njobs,
                                                    const int* __restrict__ dirty, int stage_off) {
    extern __shared__ __align__(16) float2 psm[];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ int s_fail;
    unsigned char* stage[2] = {reinterpret_cast<unsigned char*>(psm) + stage_off,
                               reinterpret_cast<unsigned char*>(psm) + stage_off + PLANE_STAGE_BYTES};
    if (threadIdx.x == 0) { sur_mbar_init(&s_bar[0]); sur_mbar_init(&s_bar[1]); s_fail = 0; }
    __syncthreads();
    auto wanted = [&](int j) { return j < njobs && (!dirty || dirty[jobs[j].x]); };
    auto issue = [&](int j, int s) {  // thread 0: the plane of job j into stage s
        const int2 job = jobs[j];
        const RepDesc& D = d.desc[job.x];
        const int n = D.mesh[0];
        int zrel = job.y - D.zb_lo;
        zrel += (zrel < 0) ? D.mesh[2] : 0;
        sur_bulk_load(stage[s], d.qband + D.qb_off + (size_t)zrel * n * n, (uint32_t)(n * n * 8), &s_bar[s]);
    };
    int uses[2] = {0, 0};  // copies issued into each stage (every thread counts alike)
    int j = blockIdx.x, it = 0;
    if (wanted(j)) { if (threadIdx.x == 0) issue(j, 0); uses[0]++; }
    for (; j < njobs; j += gridDim.x, ++it) {
        const int s = it & 1, jn = j + gridDim.x;
        if (wanted(jn)) { if (threadIdx.x == 0) issue(jn, s ^ 1); uses[s ^ 1]++; }  // its stage was read last step
        if (!wanted(j)) continue;
        if (threadIdx.x == 0 && !sur_mbar_wait(&s_bar[s], (uint32_t)((uses[s] - 1) & 1))) s_fail = 1;
        __syncthreads();
        if (s_fail) {
            if (threadIdx.x == 0) {
                atomicExch(&d.state[jobs[j].x].error, PHMC_ERR_BUDGET);
                sur_mbar_wait(&s_bar[s ^ 1], (uint32_t)((uses[s ^ 1] - 1) & 1));  // the copy in flight, bounded
            }
            return;
        }
        const int2 job = jobs[j];
        const RepDesc& D = d.desc[job.x];
        const int n = D.mesh[0];
        float2* sa = psm;
        float2* sb = psm + n * plane_ms(n / 2);
        const ulonglong2* qs = reinterpret_cast<const ulonglong2*>(stage[s]);
        switch (n) {
#define PLANE_FWD(nn, a, b) case nn: plane_fwd<nn, a, b, NT>(d, D, job.y, 0, sa, sb, qs); break;
            PLANE_LIST(PLANE_FWD)
#undef PLANE_FWD
            default: break;
        }
        __syncthreads();  // every thread is done with stage s and the plane buffers
    }
}

template <int NT>
__global__ void __launch_bounds__(NT) k_rb_inv_reg(DevPtrs d, const int2* __restrict__ jobs, const int* __restrict__ dirty) {
    extern __shared__ __align__(16) float2 psm[];
    const int2 job = jobs[blockIdx.x];
    const int r = job.x, z = job.y;
    if (dirty && !dirty[r]) return;
    const RepDesc& D = d.desc[r];
    const int n = D.mesh[0];
    float2* sa = psm;
    float2* sb = psm + n * plane_ms(n / 2);
    switch (n) {
#define PLANE_INV(nn, a, b) case nn: plane_inv<nn, a, b, NT>(d, D, z, sa, sb); break;
        PLANE_LIST(PLANE_INV)
#undef PLANE_INV
        default: break;
    }
}

bool plane_reg_supported(int nx, int ny) {
    if (nx != ny) return false;
#define PLANE_OK(nn, a, b) if (nx == nn) return true;
    PLANE_LIST(PLANE_OK)
#undef PLANE_OK
    return false;
}
size_t plane_reg_smem(int n) { return ((size_t)n * plane_ms(n / 2) + (size_t)n * (n / 2 + 1)) * sizeof(float2); }

// The unit-charge rebuild (influence kernel) computes every plane; a rebuild of the
// particles' mesh only the planes of each replica's wall band.
void launch_rebuild_r2c(Engine& E, const int* dirty, int unit_charge, cudaStream_t st) {
    const int2* pj = unit_charge ? E.d_plane_jobs : E.d_band_jobs;
    const int npj = unit_charge ? E.n_plane_jobs : E.n_band_jobs;
    if (E.plane_reg && E.fwd_pipe && !unit_charge && E.nsm > 0) {
        const int off = (int)((E.rb_fwd_smem + 127) / 128 * 128);
        const int grid = std::min(npj, 2 * E.nsm);
        k_rb_fwd_pipe<PLANE_NT><<<grid, PLANE_NT, off + 2 * PLANE_STAGE_BYTES, st>>>(E.d, pj, npj, dirty, off);
    } else if (E.plane_reg) k_rb_fwd_reg<PLANE_NT><<<npj, PLANE_NT, E.rb_fwd_smem, st>>>(E.d, pj, unit_charge, dirty);
    else k_rb_fwd<256><<<npj, 256, E.rb_fwd_smem, st>>>(E.d, pj, unit_charge, dirty);
    switch (E.zreg) {
#define ZREG_LAUNCH(id, n, a, b) \
        case id: k_rb_zreg<a, b, ZREG_NT(b), ZREG_TX><<<E.n_zjobs, ZREG_NT(b), E.zpass_smem, st>>>(E.d, E.d_zjobs, E.d_epart, dirty, unit_charge); break;
        ZREG_LIST(ZREG_LAUNCH)
#undef ZREG_LAUNCH
        default: k_rb_zpass<256, ZPASS_TX><<<E.n_zjobs, 256, E.zpass_smem, st>>>(E.d, E.d_zjobs, E.d_epart, dirty, unit_charge);
    }
    if (E.plane_reg) k_rb_inv_reg<PLANE_NT><<<npj, PLANE_NT, E.rb_inv_smem, st>>>(E.d, pj, dirty);
    else k_rb_inv<256><<<npj, 256, E.rb_inv_smem, st>>>(E.d, pj, dirty);
}

// Charge mesh of every replica's wall band from scratch (full recompute).
void launch_band_spread(Engine& E, cudaStream_t st) {
    switch (E.order) {
        case 4: k_band_spread<4, 256><<<E.n_band_jobs, 256, E.band_spread_smem, st>>>(E.d, E.d_band_jobs); break;
        case 5: k_band_spread<5, 256><<<E.n_band_jobs, 256, E.band_spread_smem, st>>>(E.d, E.d_band_jobs); break;
        default: k_band_spread<6, 256><<<E.n_band_jobs, 256, E.band_spread_smem, st>>>(E.d, E.d_band_jobs); break;
    }
}

template <typename K>
static cudaError_t raise_cap(K kernel, int device, size_t need) {
    int optin = 0;
    cudaError_t e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, kernel);
    if (e != cudaSuccess) return e;
    const int cap = optin - (int)fa.sharedSizeBytes;
    if (cap < (int)need) return cudaErrorInvalidValue;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, cap);
}

cudaError_t rebuild_set_smem_limits(Engine& E) {
    cudaError_t e = cudaSuccess;
    switch (E.order) {
        case 4: e = raise_cap(k_band_spread<4, 256>, E.device, E.band_spread_smem); break;
        case 5: e = raise_cap(k_band_spread<5, 256>, E.device, E.band_spread_smem); break;
        default: e = raise_cap(k_band_spread<6, 256>, E.device, E.band_spread_smem); break;
    }
    if (e != cudaSuccess) return e;
    e = E.plane_reg ? raise_cap(k_rb_fwd_reg<PLANE_NT>, E.device, E.rb_fwd_smem) : raise_cap(k_rb_fwd<256>, E.device, E.rb_fwd_smem);
    if (e != cudaSuccess) return e;
    if (E.nsm == 0) {
        e = cudaDeviceGetAttribute(&E.nsm, cudaDevAttrMultiProcessorCount, E.device);
        if (e != cudaSuccess) return e;
    }
    if (E.plane_reg) e = raise_cap(k_rb_fwd_pipe<PLANE_NT>, E.device, (E.rb_fwd_smem + 127) / 128 * 128 + 2 * PLANE_STAGE_BYTES);
    if (e != cudaSuccess) return e;
    switch (E.zreg) {
#define ZREG_CAP(id, n, a, b) case id: e = raise_cap(k_rb_zreg<a, b, ZREG_NT(b), ZREG_TX>, E.device, E.zpass_smem); break;
        ZREG_LIST(ZREG_CAP)
#undef ZREG_CAP
        default: e = raise_cap(k_rb_zpass<256, ZPASS_TX>, E.device, E.zpass_smem);
    }
    if (e != cudaSuccess) return e;
    return E.plane_reg ? raise_cap(k_rb_inv_reg<PLANE_NT>, E.device, E.rb_inv_smem) : raise_cap(k_rb_inv<256>, E.device, E.rb_inv_smem);
}
