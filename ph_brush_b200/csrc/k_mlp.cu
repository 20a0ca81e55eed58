// Surrogate network for the delayed-acceptance first stage: an MLP
// n_in -> H -> H -> H -> 1 with GELU, BF16 weights and activations, FP32
// accumulation on the tensor cores (mma.sync m16n8k16), trained on the GPU
// by the kernels below (forward, backward, Adam).  No counterpart in the
// reference.
//
// A training sample is one move: up to SUR_ROWS rows (the old and new state
// of each changed particle) with signs -1 / +1 (0 = unused row) and the
// target dE_env = dE - (exact terms).  The model is
//     dE_env ~ scale * sum_r sign_r y(row_r),
// the difference of a learned per-particle energy between the new and the old
// state, so the estimate of a move is minus the estimate of its reverse.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>
#include "engine.h"

// ---------------------------------------------------------------------------
// BF16 tensor-core GEMM: C[M x N] = sum_k A(i, k) B(k, j), FP32 accumulation.
// A(i,k) = A[i*sai + k*sak], B(k,j) = B[k*sbk + j*sbj] (BF16, any strides).
// Block tile 64 x 64, 4 warps of 32 x 32 (2 x 4 m16n8 tiles), K step 16.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ float gelu_grad(float x) {
    const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752440f));
    const float pdf = 0.39894228040143267794f * expf(-0.5f * x * x);
    return cdf + x * pdf;
}

enum { EPI_STORE = 0, EPI_BIAS_GELU = 1, EPI_GELU_GRAD = 2 };

// epi EPI_STORE:     Cf[i*N+j] = acc
// epi EPI_BIAS_GELU: Z = acc + bias[j] -> Cf (fp32), H = gelu(Z) -> Hb (bf16)
// epi EPI_GELU_GRAD: dZ = acc * gelu'(Zin[i*N+j]) -> Hb (bf16)
// Split K: block z covers k in [z * kchunk, min(K, (z + 1) * kchunk)) and, for EPI_STORE,
// writes its partial product to Cf + z * M * N (summed by k_sum_splits in a fixed order).
__global__ void __launch_bounds__(128) k_gemm_bf16(int M, int N, int K, const __nv_bfloat16* __restrict__ A, long sai,
                                                   long sak, const __nv_bfloat16* __restrict__ B, long sbk, long sbj,
                                                   int epi, float* __restrict__ Cf, const float* __restrict__ bias,
                                                   const float* __restrict__ Zin, __nv_bfloat16* __restrict__ Hb,
                                                   int kchunk) {
    __shared__ __nv_bfloat16 As[64][16 + 8];
    __shared__ __nv_bfloat16 Bs[16][64 + 8];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int i0 = blockIdx.y * 64, j0 = blockIdx.x * 64;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int g = lane >> 2, t4 = lane & 3;
    float acc[2][4][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.0f;
    const __nv_bfloat16 z = __float2bfloat16(0.0f);
    const int kbeg = blockIdx.z * kchunk, kend = min(K, kbeg + kchunk);
    if (epi == EPI_STORE) Cf += (size_t)blockIdx.z * M * N;
    for (int k0 = kbeg; k0 < kend; k0 += 16) {
        for (int e = tid; e < 64 * 16; e += 128) {
            const int r = e >> 4, kk = e & 15;
            const int i = i0 + r, k = k0 + kk;
            As[r][kk] = (i < M && k < kend) ? A[(long)i * sai + (long)k * sak] : z;
        }
        for (int e = tid; e < 16 * 64; e += 128) {
            const int kk = e >> 6, cc = e & 63;
            const int k = k0 + kk, j = j0 + cc;
            Bs[kk][cc] = (k < kend && j < N) ? B[(long)k * sbk + (long)j * sbj] : z;
        }
        __syncthreads();
        uint32_t af[2][4], bfr[4][2];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const int r = wm + mt * 16 + g;
            af[mt][0] = pack2(As[r][2 * t4], As[r][2 * t4 + 1]);
            af[mt][1] = pack2(As[r + 8][2 * t4], As[r + 8][2 * t4 + 1]);
            af[mt][2] = pack2(As[r][2 * t4 + 8], As[r][2 * t4 + 9]);
            af[mt][3] = pack2(As[r + 8][2 * t4 + 8], As[r + 8][2 * t4 + 9]);
        }
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const int cidx = wn + nt * 8 + g;
            bfr[nt][0] = pack2(Bs[2 * t4][cidx], Bs[2 * t4 + 1][cidx]);
            bfr[nt][1] = pack2(Bs[2 * t4 + 8][cidx], Bs[2 * t4 + 9][cidx]);
        }
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) sur_mma(acc[mt][nt], af[mt], bfr[nt][0], bfr[nt][1]);
        __syncthreads();
    }
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const int i = i0 + wm + mt * 16 + g + 8 * h;
                    const int j = j0 + wn + nt * 8 + 2 * t4 + q;
                    if (i >= M || j >= N) continue;
                    const float v = acc[mt][nt][2 * h + q];
                    const long o = (long)i * N + j;
                    if (epi == EPI_STORE) Cf[o] = v;
                    else if (epi == EPI_BIAS_GELU) {
                        const float zz = v + bias[j];
                        Cf[o] = zz;
                        Hb[o] = __float2bfloat16(sur_gelu(zz));
                    } else {
                        Hb[o] = __float2bfloat16(v * gelu_grad(Zin[o]));
                    }
                }
}

// out[i] = sum_z part[z * n + i] in z order (deterministic)
__global__ void k_sum_splits(const float* __restrict__ part, int splits, int n, float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float s = 0.0f;
    for (int z = 0; z < splits; ++z) s += part[(size_t)z * n + i];
    out[i] = s;
}

#define GEMM_MAX_SPLITS 64

// The training products run on the fifth-generation tensor cores (k_umma.cu: tcgen05.mma,
// accumulator in tensor memory) when N is at most 256; the mma.sync kernel above is the
// other path, selectable for comparison (phmc_surrogate_set_gemm).
static bool g_gemm_tcgen05 = true;

extern "C" int phmc_surrogate_set_gemm(int tcgen05) {
    g_gemm_tcgen05 = tcgen05 != 0;
    return PHMC_OK;
}

// PHMC_OK, or the error a tensor-core GEMM recorded since the last check (a bounded wait
// that ran out: its output is not written).
static int gemm_status() {
    const int e = umma_take_error(0);
    if (e) phmc_set_error(e, "surrogate GEMM: a tensor-core wait ran out (results not written)");
    return e;
}

static void gemm(int M, int N, int K, const __nv_bfloat16* A, long sai, long sak, const __nv_bfloat16* B, long sbk,
                 long sbj, int epi, float* Cf, const float* bias, const float* Zin, __nv_bfloat16* Hb, cudaStream_t st,
                 float* split_buf = nullptr) {
    const bool umma = g_gemm_tcgen05 && N <= 256;
    dim3 grid((N + 63) / 64, (M + 63) / 64, 1);
    // long-K products with few output tiles (weight gradients): split K over enough blocks to fill the GPU
    int splits = 1;
    if (epi == EPI_STORE && split_buf) {
        const int tiles = umma ? (M + 127) / 128 : (int)(grid.x * grid.y);
        splits = std::min(GEMM_MAX_SPLITS, std::max(1, (umma ? 148 : 296) / tiles));
        splits = std::min(splits, std::max(1, K / 256));
    }
    const int kchunk = ((K + splits - 1) / splits + 15) / 16 * 16;
    splits = (K + kchunk - 1) / kchunk;
    grid.z = splits;
    float* out = splits == 1 ? Cf : split_buf;
    if (umma) launch_umma_gemm(M, N, K, A, sai, sak, B, sbk, sbj, epi, out, bias, Zin, Hb, kchunk, splits, st);
    else k_gemm_bf16<<<grid, 128, 0, st>>>(M, N, K, A, sai, sak, B, sbk, sbj, epi, out, bias, Zin, Hb, kchunk);
    if (splits > 1) k_sum_splits<<<(M * N + 255) / 256, 256, 0, st>>>(split_buf, splits, M * N, Cf);
}

// ---------------------------------------------------------------------------
// small kernels
// ---------------------------------------------------------------------------
// standardised BF16 rows: row e = (sample idx[e / SUR_ROWS], row e % SUR_ROWS) when idx != null
__global__ void k_normalize(const float* __restrict__ x, const int* __restrict__ idx, long nrows, int nin,
                            const float* __restrict__ mu, const float* __restrict__ sd, __nv_bfloat16* __restrict__ out) {
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nrows * nin) return;
    const long row = e / nin;
    const int k = (int)(e - row * nin);
    const long src_row = idx ? (long)idx[row / SUR_ROWS] * SUR_ROWS + row % SUR_ROWS : row;
    out[e] = __float2bfloat16(__fdiv_rn(__fsub_rn(x[src_row * nin + k], mu[k]), sd[k]));
}

// output layer: y[i] = (h_i . w4 + b4) * scale + offset, one warp per row
__global__ void k_out_forward(const __nv_bfloat16* __restrict__ H, long n, int K, const uint16_t* __restrict__ w4,
                              const float* __restrict__ b4, float scale, float offset, float* __restrict__ y) {
    const long i = (long)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    const float v = sur_out_dot(H + i * K, w4, K, lane);
    if (lane == 0) y[i] = __fmaf_rn(v + __ldg(b4), scale, offset);
}

// per sample: pred = sum_r sign_r y_r (standardised), target clip(t)/scale;
// loss += 1/2 (pred - target)^2 / B, dy_r = sign_r (pred - target) / B
__global__ void k_loss(const float* __restrict__ y, const float* __restrict__ sign, const float* __restrict__ t,
                       const int* __restrict__ idx, int B, float scale, float clip, float* __restrict__ dy,
                       double* __restrict__ loss) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.0;
    if (i < B) {
        const long s = idx ? idx[i] : i;
        float pred = 0.0f, sg[SUR_ROWS];
#pragma unroll
        for (int r = 0; r < SUR_ROWS; ++r) {
            sg[r] = sign[s * SUR_ROWS + r];
            pred += sg[r] * y[(long)i * SUR_ROWS + r];
        }
        const float tt = fminf(fmaxf(t[s], -clip), clip) / scale;
        const float dd = pred - tt;
#pragma unroll
        for (int r = 0; r < SUR_ROWS; ++r) dy[(long)i * SUR_ROWS + r] = sg[r] * dd / (float)B;
        l = 0.5 * (double)dd * dd / B;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}

// output layer backward: dZ3 = dy w4 * gelu'(Z3) (bf16)
__global__ void k_out_backward(const float* __restrict__ dy, const float* __restrict__ Z, long n, int K,
                               const uint16_t* __restrict__ w4, __nv_bfloat16* __restrict__ dZ) {
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * K) return;
    const long i = e / K;
    const int k = (int)(e - i * K);
    dZ[e] = __float2bfloat16(dy[i] * __bfloat162float(__ushort_as_bfloat16(w4[k])) * gelu_grad(Z[e]));
}

// dw4[k] = sum_i dy_i h_ik, db4 = sum_i dy_i (block K handles the bias)
__global__ void k_out_wgrad(const float* __restrict__ dy, const __nv_bfloat16* __restrict__ H, long n, int K,
                            float* __restrict__ gw, float* __restrict__ gb) {
    const int k = blockIdx.x;
    float s = 0.0f;
    for (long i = threadIdx.x; i < n; i += blockDim.x) s += dy[i] * (k < K ? __bfloat162float(H[i * K + k]) : 1.0f);
    __shared__ float red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float tot = 0.0f;
        for (int w = 0; w < (int)blockDim.x / 32; ++w) tot += red[w];
        if (k < K) gw[k] = tot; else *gb = tot;
    }
}

// column sums of a bf16 matrix (bias gradients)
__global__ void k_colsum(const __nv_bfloat16* __restrict__ X, long n, int N, float* __restrict__ out) {
    const int j = blockIdx.x;
    float s = 0.0f;
    for (long i = threadIdx.x; i < n; i += blockDim.x) s += __bfloat162float(X[i * N + j]);
    __shared__ float red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float tot = 0.0f;
        for (int w = 0; w < (int)blockDim.x / 32; ++w) tot += red[w];
        out[j] = tot;
    }
}

// Adam (Kingma & Ba 2015) on the FP32 master copy, then the BF16 working copy.
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v, int n,
                       float lr, float b1, float b2, float eps, float c1, float c2, __nv_bfloat16* __restrict__ pb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi; v[i] = vi;
    const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    pb[i] = __float2bfloat16(pi);
}

__global__ void k_f32_to_bf16(const float* __restrict__ a, __nv_bfloat16* __restrict__ b, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = __float2bfloat16(a[i]);
}

// mean / standard deviation of every feature over the rows with a non-zero sign
// (one block per feature; sd = 1 for a feature that does not vary)
__global__ void k_feature_stats(const float* __restrict__ x, const float* __restrict__ sign, long nrows, int nin,
                                float* __restrict__ mu, float* __restrict__ sd) {
    const int k = blockIdx.x;
    double s = 0.0, s2 = 0.0, c = 0.0;
    for (long r = threadIdx.x; r < nrows; r += blockDim.x) {
        if (sign[r] == 0.0f) continue;
        const double v = x[r * nin + k];
        s += v; s2 += v * v; c += 1.0;
    }
    __shared__ double red[3][32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = s; red[1][threadIdx.x >> 5] = s2; red[2][threadIdx.x >> 5] = c; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0, n = 0;
        for (int w = 0; w < (int)blockDim.x / 32; ++w) { a += red[0][w]; b += red[1][w]; n += red[2][w]; }
        const double m = n > 0 ? a / n : 0.0;
        const double var = n > 0 ? b / n - m * m : 0.0;
        mu[k] = (float)m;
        sd[k] = var > 1e-6 ? (float)sqrt(var) : 1.0f;
    }
}

// root mean square of the clipped targets (one block)
__global__ void k_target_rms(const float* __restrict__ t, int n, float clip, float* __restrict__ out) {
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double v = fmin(fmax((double)t[i], -(double)clip), (double)clip);
        s += v * v;
    }
    __shared__ double red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0;
        for (int w = 0; w < (int)blockDim.x / 32; ++w) a += red[w];
        const double rms = n > 0 ? sqrt(a / n) : 0.0;
        *out = rms > 1e-3 ? (float)rms : 1.0f;
    }
}

// K x H row-major FP32 matrix -> fragment-packed BF16 (sur_pack_index), rows >= K zero
__global__ void k_pack_frag(const float* __restrict__ W, int K, int Kp, int H, uint2* __restrict__ out) {
    const int nks = Kp / 16;
    const int total = (H / 16) * nks * 2 * 32;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const int lane = e & 31, nt = (e >> 5) & 1;
    const int ks = (e >> 6) % nks, cg = (e >> 6) / nks;
    const int n = cg * 16 + nt * 8 + (lane >> 2);
    const int k0 = ks * 16 + 2 * (lane & 3);
    auto w = [&](int k) { return __float2bfloat16(k < K ? W[(size_t)k * H + n] : 0.0f); };
    out[sur_pack_index(cg, ks, nt, lane, nks)] = make_uint2(pack2(w(k0), w(k0 + 1)), pack2(w(k0 + 8), w(k0 + 9)));
}

// ---------------------------------------------------------------------------
// host object
// ---------------------------------------------------------------------------
struct phmc_surrogate {
    int nin = 0, H = 0, nparam = 0;
    int off[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    float* p = nullptr;                 // FP32 master parameters
    __nv_bfloat16* pb = nullptr;        // BF16 working copy (same layout)
    float* mu = nullptr;                // input standardisation [nin]
    float* sd = nullptr;
    float scale = 1.0f;                 // energy = scale * y
    uint2* packed[3] = {nullptr, nullptr, nullptr};  // fragment-packed hidden layers
    bool packed_ok = false;
    long cap = 0;                       // row capacity of the activation buffers
    __nv_bfloat16* X = nullptr;
    float* Z[3] = {nullptr, nullptr, nullptr};
    __nv_bfloat16* Hb[3] = {nullptr, nullptr, nullptr};
    __nv_bfloat16* dZ[3] = {nullptr, nullptr, nullptr};
    float *y = nullptr, *dy = nullptr;
    double* loss = nullptr;
    float* grad = nullptr;
    float *adam_m = nullptr, *adam_v = nullptr;
    float* d_scale = nullptr;
    float* split = nullptr;             // split-K partial products (GEMM_MAX_SPLITS x max(n_in, H) x H)
    int adam_t = 0;
    std::vector<void*> allocs;
};

#define MCU(x)                                                                                     \
    do {                                                                                           \
        cudaError_t e_ = (x);                                                                      \
        if (e_ != cudaSuccess) { phmc_set_error(PHMC_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); return PHMC_ERR_CUDA; } \
    } while (0)

template <typename T>
static int malloc_t(phmc_surrogate* h, T** p, size_t n) {
    MCU(cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(n, 1)));
    h->allocs.push_back(*p);
    return PHMC_OK;
}

static void free_t(phmc_surrogate* h, void* p) {
    if (!p) return;
    cudaFree(p);
    h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), p), h->allocs.end());
}

// parameter layout (FP32 master, flat): W1[nin*H], b1[H], W2[H*H], b2[H], W3[H*H], b3[H], w4[H], b4[1];
// W[k*H + j] connects input k to output j
static void layout(int nin, int H, int off[8], int* total) {
    int o = 0;
    off[0] = o; o += nin * H;
    off[1] = o; o += H;
    off[2] = o; o += H * H;
    off[3] = o; o += H;
    off[4] = o; o += H * H;
    off[5] = o; o += H;
    off[6] = o; o += H;
    off[7] = o; o += 1;
    *total = o;
}

static int ensure_rows(phmc_surrogate* h, long n) {
    if (n <= h->cap) return PHMC_OK;
    void* old[] = {h->X, h->Z[0], h->Z[1], h->Z[2], h->Hb[0], h->Hb[1], h->Hb[2], h->dZ[0], h->dZ[1], h->dZ[2], h->y, h->dy};
    for (void* p : old) free_t(h, p);
    h->cap = 0;
    const long c = std::max(n, 4096L);
    int s;
    if ((s = malloc_t(h, &h->X, (size_t)c * h->nin))) return s;
    for (int l = 0; l < 3; ++l) {
        if ((s = malloc_t(h, &h->Z[l], (size_t)c * h->H))) return s;
        if ((s = malloc_t(h, &h->Hb[l], (size_t)c * h->H))) return s;
        if ((s = malloc_t(h, &h->dZ[l], (size_t)c * h->H))) return s;
    }
    if ((s = malloc_t(h, &h->y, c))) return s;
    if ((s = malloc_t(h, &h->dy, c))) return s;
    h->cap = c;
    return PHMC_OK;
}

extern "C" int phmc_surrogate_create(int n_in, int hidden, uint64_t seed, phmc_surrogate** out) {
    if (!out || n_in < 1 || n_in > 4 * SUR_K || hidden < 16 || hidden > SUR_HMAX || hidden % 16) {
        phmc_set_error(PHMC_ERR_ARG, "phmc_surrogate_create: 1 <= n_in <= 320 and hidden a multiple of 16 in [16, 128]");
        return PHMC_ERR_ARG;
    }
    *out = nullptr;
    phmc_surrogate* h = new phmc_surrogate;
    h->nin = n_in;
    h->H = hidden;
    layout(n_in, hidden, h->off, &h->nparam);
    std::vector<float> p((size_t)h->nparam, 0.0f);
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.0f, 1.0f);
    auto init = [&](int o, int fan_in, int count, float gain) {  // He-normal for the GELU layers
        const float s = gain * std::sqrt(2.0f / fan_in);
        for (int i = 0; i < count; ++i) p[(size_t)o + i] = s * nd(rng);
    };
    init(h->off[0], n_in, n_in * hidden, 1.0f);
    init(h->off[2], hidden, hidden * hidden, 1.0f);
    init(h->off[4], hidden, hidden * hidden, 1.0f);
    init(h->off[6], hidden, hidden, 0.5f);
    int s = 0;
    const int nk1 = (n_in + 15) / 16 * 16;
    if ((s = malloc_t(h, &h->p, h->nparam)) || (s = malloc_t(h, &h->pb, h->nparam)) || (s = malloc_t(h, &h->grad, h->nparam)) ||
        (s = malloc_t(h, &h->adam_m, h->nparam)) || (s = malloc_t(h, &h->adam_v, h->nparam)) ||
        (s = malloc_t(h, &h->mu, n_in)) || (s = malloc_t(h, &h->sd, n_in)) || (s = malloc_t(h, &h->loss, 1)) ||
        (s = malloc_t(h, &h->d_scale, 1)) || (s = malloc_t(h, &h->packed[0], (size_t)nk1 * hidden / 4)) ||
        (s = malloc_t(h, &h->split, (size_t)GEMM_MAX_SPLITS * std::max(n_in, hidden) * hidden)) ||
        (s = malloc_t(h, &h->packed[1], (size_t)hidden * hidden / 4)) || (s = malloc_t(h, &h->packed[2], (size_t)hidden * hidden / 4))) {
        phmc_surrogate_destroy(h);
        return s;
    }
    std::vector<float> mu((size_t)n_in, 0.0f), sd((size_t)n_in, 1.0f);
    cudaMemcpy(h->p, p.data(), sizeof(float) * p.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(h->mu, mu.data(), sizeof(float) * mu.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(h->sd, sd.data(), sizeof(float) * sd.size(), cudaMemcpyHostToDevice);
    cudaMemset(h->adam_m, 0, sizeof(float) * h->nparam);
    cudaMemset(h->adam_v, 0, sizeof(float) * h->nparam);
    k_f32_to_bf16<<<(h->nparam + 255) / 256, 256>>>(h->p, h->pb, h->nparam);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) { phmc_set_error(PHMC_ERR_CUDA, cudaGetErrorString(e)); phmc_surrogate_destroy(h); return PHMC_ERR_CUDA; }
    *out = h;
    return PHMC_OK;
}

extern "C" int phmc_surrogate_destroy(phmc_surrogate* h) {
    if (!h) return PHMC_OK;
    cudaDeviceSynchronize();
    for (void* p : h->allocs) cudaFree(p);
    delete h;
    return PHMC_OK;
}

// Forward pass over n rows already standardised in h->X; y = scale * out + offset.
static void forward_rows(phmc_surrogate* h, long n, float scale, float offset, cudaStream_t st) {
    const int H = h->H, nin = h->nin;
    const __nv_bfloat16* W = h->pb;
    const int* off = h->off;
    gemm((int)n, H, nin, h->X, nin, 1, W + off[0], H, 1, EPI_BIAS_GELU, h->Z[0], h->p + off[1], nullptr, h->Hb[0], st);
    gemm((int)n, H, H, h->Hb[0], H, 1, W + off[2], H, 1, EPI_BIAS_GELU, h->Z[1], h->p + off[3], nullptr, h->Hb[1], st);
    gemm((int)n, H, H, h->Hb[1], H, 1, W + off[4], H, 1, EPI_BIAS_GELU, h->Z[2], h->p + off[5], nullptr, h->Hb[2], st);
    k_out_forward<<<(int)((n + 3) / 4), 128, 0, st>>>(h->Hb[2], n, H, reinterpret_cast<const uint16_t*>(W + off[6]),
                                                       h->p + off[7], scale, offset, h->y);
}

// Backward of the signed-row loss over B samples (B * SUR_ROWS rows already
// forwarded); accumulates the loss into h->loss, leaves the gradient in h->grad.
static void backward_rows(phmc_surrogate* h, const float* d_sign, const float* d_t, const int* d_idx, int B, float clip,
                          cudaStream_t st) {
    const int H = h->H, nin = h->nin;
    const __nv_bfloat16* W = h->pb;
    const int* off = h->off;
    const long n = (long)B * SUR_ROWS;
    k_loss<<<(B + 255) / 256, 256, 0, st>>>(h->y, d_sign, d_t, d_idx, B, h->scale, clip, h->dy, h->loss);
    k_out_wgrad<<<H + 1, 256, 0, st>>>(h->dy, h->Hb[2], n, H, h->grad + off[6], h->grad + off[7]);
    k_out_backward<<<(int)((n * H + 255) / 256), 256, 0, st>>>(h->dy, h->Z[2], n, H, reinterpret_cast<const uint16_t*>(W + off[6]), h->dZ[2]);
    // layer 3: dW3 = H2^T dZ3, db3 = colsum dZ3, dZ2 = (dZ3 W3^T) * gelu'(Z2)
    gemm(H, H, (int)n, h->Hb[1], 1, H, h->dZ[2], H, 1, EPI_STORE, h->grad + off[4], nullptr, nullptr, nullptr, st, h->split);
    k_colsum<<<H, 256, 0, st>>>(h->dZ[2], n, H, h->grad + off[5]);
    gemm((int)n, H, H, h->dZ[2], H, 1, W + off[4], 1, H, EPI_GELU_GRAD, nullptr, nullptr, h->Z[1], h->dZ[1], st);
    // layer 2
    gemm(H, H, (int)n, h->Hb[0], 1, H, h->dZ[1], H, 1, EPI_STORE, h->grad + off[2], nullptr, nullptr, nullptr, st, h->split);
    k_colsum<<<H, 256, 0, st>>>(h->dZ[1], n, H, h->grad + off[3]);
    gemm((int)n, H, H, h->dZ[1], H, 1, W + off[2], 1, H, EPI_GELU_GRAD, nullptr, nullptr, h->Z[0], h->dZ[0], st);
    // layer 1
    gemm(nin, H, (int)n, h->X, 1, nin, h->dZ[0], H, 1, EPI_STORE, h->grad + off[0], nullptr, nullptr, nullptr, st, h->split);
    k_colsum<<<H, 256, 0, st>>>(h->dZ[0], n, H, h->grad + off[1]);
}

extern "C" int phmc_surrogate_set_scaling(phmc_surrogate* h, const float* mu, const float* sd, float scale) {
    if (!h || !mu || !sd || !(scale > 0)) { phmc_set_error(PHMC_ERR_ARG, "phmc_surrogate_set_scaling: bad argument"); return PHMC_ERR_ARG; }
    for (int k = 0; k < h->nin; ++k)
        if (!(sd[k] > 0)) { phmc_set_error(PHMC_ERR_ARG, "phmc_surrogate_set_scaling: sd must be > 0"); return PHMC_ERR_ARG; }
    MCU(cudaMemcpy(h->mu, mu, sizeof(float) * h->nin, cudaMemcpyHostToDevice));
    MCU(cudaMemcpy(h->sd, sd, sizeof(float) * h->nin, cudaMemcpyHostToDevice));
    h->scale = scale;
    return PHMC_OK;
}

extern "C" int phmc_surrogate_get_scaling(phmc_surrogate* h, float* mu, float* sd, float* scale) {
    if (!h) { phmc_set_error(PHMC_ERR_ARG, "null surrogate"); return PHMC_ERR_ARG; }
    if (mu) MCU(cudaMemcpy(mu, h->mu, sizeof(float) * h->nin, cudaMemcpyDeviceToHost));
    if (sd) MCU(cudaMemcpy(sd, h->sd, sizeof(float) * h->nin, cudaMemcpyDeviceToHost));
    if (scale) *scale = h->scale;
    return PHMC_OK;
}

extern "C" int phmc_surrogate_num_params(phmc_surrogate* h) { return h ? h->nparam : -1; }

extern "C" int phmc_surrogate_get_params(phmc_surrogate* h, float* out, int n) {
    if (!h || !out || n < h->nparam) { phmc_set_error(PHMC_ERR_ARG, "phmc_surrogate_get_params: buffer too small"); return PHMC_ERR_ARG; }
    MCU(cudaMemcpy(out, h->p, sizeof(float) * h->nparam, cudaMemcpyDeviceToHost));
    return PHMC_OK;
}

extern "C" int phmc_surrogate_set_params(phmc_surrogate* h, const float* in, int n) {
    if (!h || !in || n != h->nparam) { phmc_set_error(PHMC_ERR_ARG, "phmc_surrogate_set_params: size mismatch"); return PHMC_ERR_ARG; }
    MCU(cudaMemcpy(h->p, in, sizeof(float) * n, cudaMemcpyHostToDevice));
    k_f32_to_bf16<<<(n + 255) / 256, 256>>>(h->p, h->pb, n);
    MCU(cudaDeviceSynchronize());
    h->packed_ok = false;
    return PHMC_OK;
}

// predictions (energy units) for n host rows
extern "C" int phmc_surrogate_predict(phmc_surrogate* h, const float* x, int n, float* y) {
    if (!h || (n > 0 && (!x || !y))) { phmc_set_error(PHMC_ERR_ARG, "phmc_surrogate_predict: null argument"); return PHMC_ERR_ARG; }
    if (n == 0) return PHMC_OK;
    int s = ensure_rows(h, n);
    if (s) return s;
    float* dx = nullptr;
    MCU(cudaMalloc(&dx, sizeof(float) * (size_t)n * h->nin));
    cudaMemcpy(dx, x, sizeof(float) * (size_t)n * h->nin, cudaMemcpyHostToDevice);
    k_normalize<<<(int)(((long)n * h->nin + 255) / 256), 256>>>(dx, nullptr, n, h->nin, h->mu, h->sd, h->X);
    forward_rows(h, n, h->scale, 0.0f, 0);
    cudaError_t e = cudaMemcpy(y, h->y, sizeof(float) * n, cudaMemcpyDeviceToHost);
    cudaFree(dx);
    if (e != cudaSuccess) { phmc_set_error(PHMC_ERR_CUDA, cudaGetErrorString(e)); return PHMC_ERR_CUDA; }
    return gemm_status();
}

// loss and gradient (w.r.t. the flat master parameters) of n host samples with the current scaling
extern "C" int phmc_surrogate_gradient(phmc_surrogate* h, const float* x, const float* sign, const float* t, int n, float clip,
                                       double* loss, float* grad) {
    if (!h || !x || !sign || !t || !loss || !grad || n < 1 || !(clip > 0)) {
        phmc_set_error(PHMC_ERR_ARG, "phmc_surrogate_gradient: bad argument");
        return PHMC_ERR_ARG;
    }
    const long rows = (long)n * SUR_ROWS;
    int s = ensure_rows(h, rows);
    if (s) return s;
    float *dx = nullptr, *ds = nullptr, *dt = nullptr;
    MCU(cudaMalloc(&dx, sizeof(float) * (size_t)rows * h->nin));
    MCU(cudaMalloc(&ds, sizeof(float) * (size_t)rows));
    MCU(cudaMalloc(&dt, sizeof(float) * n));
    cudaMemcpy(dx, x, sizeof(float) * (size_t)rows * h->nin, cudaMemcpyHostToDevice);
    cudaMemcpy(ds, sign, sizeof(float) * rows, cudaMemcpyHostToDevice);
    cudaMemcpy(dt, t, sizeof(float) * n, cudaMemcpyHostToDevice);
    k_normalize<<<(int)((rows * h->nin + 255) / 256), 256>>>(dx, nullptr, rows, h->nin, h->mu, h->sd, h->X);
    forward_rows(h, rows, 1.0f, 0.0f, 0);
    cudaMemset(h->loss, 0, sizeof(double));
    backward_rows(h, ds, dt, nullptr, n, clip, 0);
    cudaError_t e = cudaMemcpy(grad, h->grad, sizeof(float) * h->nparam, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(loss, h->loss, sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(dx); cudaFree(ds); cudaFree(dt);
    if (e != cudaSuccess) { phmc_set_error(PHMC_ERR_CUDA, cudaGetErrorString(e)); return PHMC_ERR_CUDA; }
    return gemm_status();
}

// Adam training on device-resident samples (rows [ns][SUR_ROWS][nin], signs, targets).
// rescale: first set the input standardisation and the output scale from the data.
int sur_train_device(phmc_surrogate* h, const float* d_x, const float* d_sign, const float* d_t, int ns, int epochs,
                     int batch, float lr, float clip, uint64_t seed, int rescale, double* last_loss) {
    if (ns < batch || batch < 1 || epochs < 0 || !(clip > 0) || !(lr > 0)) {
        phmc_set_error(PHMC_ERR_ARG, "surrogate training: need n_samples >= batch >= 1, clip > 0, lr > 0");
        return PHMC_ERR_ARG;
    }
    int s = ensure_rows(h, (long)batch * SUR_ROWS);
    if (s) return s;
    if (rescale) {
        k_feature_stats<<<h->nin, 256>>>(d_x, d_sign, (long)ns * SUR_ROWS, h->nin, h->mu, h->sd);
        k_target_rms<<<1, 1024>>>(d_t, ns, clip, h->d_scale);
        MCU(cudaMemcpy(&h->scale, h->d_scale, sizeof(float), cudaMemcpyDeviceToHost));
    }
    std::mt19937_64 rng(seed);
    std::vector<int> perm((size_t)ns);
    for (int i = 0; i < ns; ++i) perm[(size_t)i] = i;
    int* d_perm = nullptr;
    MCU(cudaMalloc(&d_perm, sizeof(int) * (size_t)ns));
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    double lsum = 0.0;
    int nb = 0;
    for (int ep = 0; ep < epochs; ++ep) {
        std::shuffle(perm.begin(), perm.end(), rng);
        cudaMemcpy(d_perm, perm.data(), sizeof(int) * (size_t)ns, cudaMemcpyHostToDevice);
        cudaMemset(h->loss, 0, sizeof(double));
        nb = 0;
        for (int b0 = 0; b0 + batch <= ns; b0 += batch) {
            const int* idx = d_perm + b0;
            const long rows = (long)batch * SUR_ROWS;
            k_normalize<<<(int)((rows * h->nin + 255) / 256), 256>>>(d_x, idx, rows, h->nin, h->mu, h->sd, h->X);
            forward_rows(h, rows, 1.0f, 0.0f, 0);
            backward_rows(h, d_sign, d_t, idx, batch, clip, 0);
            ++h->adam_t;
            const float c1 = 1.0f - std::pow(b1, (float)h->adam_t), c2 = 1.0f - std::pow(b2, (float)h->adam_t);
            k_adam<<<(h->nparam + 255) / 256, 256>>>(h->p, h->grad, h->adam_m, h->adam_v, h->nparam, lr, b1, b2, eps, c1, c2, h->pb);
            ++nb;
        }
        MCU(cudaMemcpy(&lsum, h->loss, sizeof(double), cudaMemcpyDeviceToHost));
    }
    cudaError_t e = cudaDeviceSynchronize();
    cudaFree(d_perm);
    if (e != cudaSuccess) { phmc_set_error(PHMC_ERR_CUDA, cudaGetErrorString(e)); return PHMC_ERR_CUDA; }
    h->packed_ok = false;
    s = gemm_status();
    if (s) return s;
    if (last_loss) *last_loss = nb ? lsum / nb : 0.0;
    return PHMC_OK;
}

extern "C" int phmc_surrogate_train(phmc_surrogate* h, const float* x, const float* sign, const float* t, int n, int epochs,
                                    int batch, float lr, float clip, uint64_t seed, int rescale, double* last_loss) {
    if (!h || !x || !sign || !t || n < 1) { phmc_set_error(PHMC_ERR_ARG, "phmc_surrogate_train: bad argument"); return PHMC_ERR_ARG; }
    const size_t rows = (size_t)n * SUR_ROWS;
    float *dx = nullptr, *ds = nullptr, *dt = nullptr;
    MCU(cudaMalloc(&dx, sizeof(float) * rows * h->nin));
    MCU(cudaMalloc(&ds, sizeof(float) * rows));
    MCU(cudaMalloc(&dt, sizeof(float) * n));
    cudaMemcpy(dx, x, sizeof(float) * rows * h->nin, cudaMemcpyHostToDevice);
    cudaMemcpy(ds, sign, sizeof(float) * rows, cudaMemcpyHostToDevice);
    cudaMemcpy(dt, t, sizeof(float) * n, cudaMemcpyHostToDevice);
    const int s = sur_train_device(h, dx, ds, dt, n, epochs, batch, lr, clip, seed, rescale, last_loss);
    cudaFree(dx); cudaFree(ds); cudaFree(dt);
    return s;
}

// Device view for in-kernel inference (packs the hidden layers when they changed).
int sur_device_view(phmc_surrogate* h, SurDev* out) {
    if (h->nin != SUR_K || h->H % 16 || h->H > SUR_HMAX) {
        phmc_set_error(PHMC_ERR_UNSUPPORTED, "the engine's first stage needs n_in == 80 and hidden a multiple of 16 <= 128");
        return PHMC_ERR_UNSUPPORTED;
    }
    if (!h->packed_ok) {
        const int Ks[3] = {h->nin, h->H, h->H};
        const int offs[3] = {h->off[0], h->off[2], h->off[4]};
        for (int l = 0; l < 3; ++l) {
            const int Kp = (Ks[l] + 15) / 16 * 16;
            const int total = (h->H / 16) * (Kp / 16) * 64;
            k_pack_frag<<<(total + 255) / 256, 256>>>(h->p + offs[l], Ks[l], Kp, h->H, h->packed[l]);
        }
        MCU(cudaDeviceSynchronize());
        h->packed_ok = true;
    }
    std::memset(out, 0, sizeof(*out));
    for (int l = 0; l < 3; ++l) out->w[l] = h->packed[l];
    out->b[0] = h->p + h->off[1]; out->b[1] = h->p + h->off[3]; out->b[2] = h->p + h->off[5];
    out->w4 = reinterpret_cast<const uint16_t*>(h->pb + h->off[6]);
    out->b4 = h->p + h->off[7];
    out->mu = h->mu; out->sd = h->sd;
    out->scale = h->scale; out->offset = 0.0f;
    out->H = h->H;
    return PHMC_OK;
}

extern "C" int phmc_surrogate_save(phmc_surrogate* h, const char* path) {
    if (!h || !path) { phmc_set_error(PHMC_ERR_ARG, "phmc_surrogate_save: null argument"); return PHMC_ERR_ARG; }
    std::vector<float> p((size_t)h->nparam), mu((size_t)h->nin), sd((size_t)h->nin);
    MCU(cudaMemcpy(p.data(), h->p, sizeof(float) * p.size(), cudaMemcpyDeviceToHost));
    MCU(cudaMemcpy(mu.data(), h->mu, sizeof(float) * mu.size(), cudaMemcpyDeviceToHost));
    MCU(cudaMemcpy(sd.data(), h->sd, sizeof(float) * sd.size(), cudaMemcpyDeviceToHost));
    FILE* f = fopen(path, "wb");
    if (!f) { phmc_set_error(PHMC_ERR_IO, std::string("cannot write ") + path); return PHMC_ERR_IO; }
    const int hdr[4] = {0x31535048 /* "HPS1" */, h->nin, h->H, h->nparam};
    bool ok = fwrite(hdr, sizeof(int), 4, f) == 4 && fwrite(&h->scale, sizeof(float), 1, f) == 1 &&
              fwrite(mu.data(), sizeof(float), mu.size(), f) == mu.size() && fwrite(sd.data(), sizeof(float), sd.size(), f) == sd.size() &&
              fwrite(p.data(), sizeof(float), p.size(), f) == p.size();
    ok = (fclose(f) == 0) && ok;
    if (!ok) { phmc_set_error(PHMC_ERR_IO, std::string("short write to ") + path); return PHMC_ERR_IO; }
    return PHMC_OK;
}

extern "C" int phmc_surrogate_load(const char* path, phmc_surrogate** out) {
    if (!path || !out) { phmc_set_error(PHMC_ERR_ARG, "phmc_surrogate_load: null argument"); return PHMC_ERR_ARG; }
    *out = nullptr;
    FILE* f = fopen(path, "rb");
    if (!f) { phmc_set_error(PHMC_ERR_IO, std::string("cannot read ") + path); return PHMC_ERR_IO; }
    int hdr[4] = {0, 0, 0, 0};
    float sc = 1.0f;
    if (fread(hdr, sizeof(int), 4, f) != 4 || hdr[0] != 0x31535048 || fread(&sc, sizeof(float), 1, f) != 1 || hdr[1] < 1 ||
        hdr[1] > 4 * SUR_K || hdr[2] < 16 || hdr[2] > SUR_HMAX) {
        fclose(f);
        phmc_set_error(PHMC_ERR_IO, std::string("not a surrogate file: ") + path);
        return PHMC_ERR_IO;
    }
    phmc_surrogate* h = nullptr;
    int s = phmc_surrogate_create(hdr[1], hdr[2], 0, &h);
    if (s) { fclose(f); return s; }
    std::vector<float> mu((size_t)hdr[1]), sd((size_t)hdr[1]), p((size_t)std::max(hdr[3], 0));
    const bool ok = hdr[3] == h->nparam && fread(mu.data(), 4, mu.size(), f) == mu.size() &&
                    fread(sd.data(), 4, sd.size(), f) == sd.size() && fread(p.data(), 4, p.size(), f) == p.size();
    fclose(f);
    if (!ok) { phmc_surrogate_destroy(h); phmc_set_error(PHMC_ERR_IO, std::string("truncated surrogate file: ") + path); return PHMC_ERR_IO; }
    if ((s = phmc_surrogate_set_scaling(h, mu.data(), sd.data(), sc)) || (s = phmc_surrogate_set_params(h, p.data(), (int)p.size()))) {
        phmc_surrogate_destroy(h);
        return s;
    }
    *out = h;
    return PHMC_OK;
}
