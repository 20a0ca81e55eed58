// Fifth-generation tensor-core GEMM (tcgen05 / UMMA, sm_100a) for the surrogate's
// training products: C[M x N] = sum_k A(i, k) B(k, j), BF16 operands, FP32
// accumulation in tensor memory.  Same operand strides, epilogues and split-K
// contract as the mma.sync GEMM in k_mlp.cu (A(i,k) = A[i*sai + k*sak],
// B(k,j) = B[k*sbk + j*sbj]); no counterpart in the reference.
//
// One CTA of 128 threads per 128-row tile of C and all N <= 256 columns:
//  * K advances in chunks of 64 through two shared-memory stages; all threads
//    stage a chunk of A (128 x 64) and B (N x 64) in the canonical K-major
//    layout without swizzle (8-row x 16-byte core matrices, 128 bytes each,
//    consecutive in the M / N direction, the next 8 columns of K one
//    "leading byte offset" further): 16-byte cp.async where the operand is
//    contiguous along K, a warp-wide movmatrix transpose of 8 x 8 blocks
//    where it is contiguous along M / N;
//  * one thread issues the chunk's four 128 x N x 16 MMAs (tcgen05.mma
//    .cta_group::1.kind::f16, smem descriptors for A and B, accumulator in
//    TMEM) and commits them to the stage's mbarrier, which frees the stage
//    for the chunk after next;
//  * the epilogue reads the accumulator with tcgen05.ld (each warp its 32
//    TMEM lanes = rows) into a shared-memory tile, then applies the GEMM's
//    epilogue and stores C along the rows.
// Every wait on an mbarrier is bounded; a wait that runs out records
// PHMC_ERR_BUDGET in *err, the CTA then waits (bounded) for its MMAs in flight,
// frees its tensor memory and returns.
#include <cstdint>
#include "engine.h"

namespace {

constexpr int UM_KC = 64;      // K per stage
constexpr int UM_ROWS = 128;   // M per CTA (one TMEM lane per row)
constexpr uint32_t UM_WAIT = 1u << 22;

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: start address, leading (K-direction) and stride
// (M/N-direction) byte offsets in 16-byte units, descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t umma_sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major, M x N.
__device__ __forceinline__ uint32_t umma_idesc(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* b) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(b)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity) {
    for (uint32_t it = 0; it < UM_WAIT; ++it) {
        uint32_t ok;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(ok)
                     : "r"(su32(b)), "r"(parity)
                     : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void umma_issue(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    const uint32_t z = 0;
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n"
        :
        : "r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* b) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(b)) : "memory");
}

__device__ __forceinline__ float gelu_dev(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752440f)); }
__device__ __forceinline__ float gelu_grad_dev(float x) {
    const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752440f));
    const float pdf = 0.39894228040143267794f * expf(-0.5f * x * x);
    return cdf + x * pdf;
}

// Stage one K chunk of `rows` rows (element (r, k) = src[(row0 + r) * s_r + (k0 + k) * s_k], zero
// outside [0, nrow) x [k0, kend)) into the canonical K-major layout at dst: 8-row x 16-byte core
// matrices of 128 bytes, consecutive along the rows, the next 8 columns of K one
// (rows / 8) x 128 bytes further.  Every load of a chunk is in flight before the chunk is
// waited for:
//  * contiguous along K (s_k == 1, 16-byte aligned rows): one 16-byte cp.async per core-matrix
//    row (zero-filled outside the tile); groups that straddle kend go element by element;
//  * contiguous along the rows (s_r == 1): each warp moves whole core matrices — lane i loads
//    the two elements (rows 2(i%4), 2(i%4)+1) of K column i/4 as one 4-byte word (the 8 x 8
//    block in movmatrix's fragment layout, K along its rows), movmatrix.trans hands lane i
//    K columns 2(i%4), 2(i%4)+1 of row i/4, which is the 4-byte word at byte 4i of the core
//    matrix; 32 blocks' loads are issued before the first transpose;
//  * anything else element by element.
// The caller completes the cp.asyncs (cp.async.wait_all) before the tensor cores read.
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(su32(sdst)), "l"(gsrc), "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ uint32_t movmatrix_t(uint32_t a) {
    uint32_t d;
    asm volatile("movmatrix.sync.aligned.m8n8.trans.b16 %0, %1;" : "=r"(d) : "r"(a));
    return d;
}

__device__ __forceinline__ void stage_tile(unsigned char* dst, int rows, const __nv_bfloat16* __restrict__ src,
                                           long s_r, long s_k, int row0, int nrow, int k0, int kend) {
    const __nv_bfloat16 z = __float2bfloat16(0.0f);
    const int groups = rows >> 3;
    auto put = [&](int r, int k, __nv_bfloat16 v) {
        *reinterpret_cast<__nv_bfloat16*>(dst + ((((k >> 3) * groups + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1))) = v;
    };
    auto get = [&](int r, int k) {
        const int gr = row0 + r, gk = k0 + k;
        return (gr < nrow && gk < kend) ? src[(long)gr * s_r + (long)gk * s_k] : z;
    };
    if (s_k == 1 && ((uintptr_t)src & 15) == 0 && (s_r & 7) == 0) {
        for (int g = threadIdx.x; g < rows * (UM_KC / 8); g += blockDim.x) {
            const int r = g / (UM_KC / 8), kq = (g - r * (UM_KC / 8)) * 8;
            const int gr = row0 + r, gk = k0 + kq;
            unsigned char* d = dst + ((((kq >> 3) * groups + (r >> 3)) << 7) + ((r & 7) << 4));
            if (gr < nrow && gk < kend && gk + 8 > kend) {
                union { uint4 u; __nv_bfloat16 h[8]; } v;  // 16-byte aligned either way
                for (int q = 0; q < 8; ++q) v.h[q] = get(r, kq + q);
                *reinterpret_cast<uint4*>(d) = v.u;
            } else {
                const bool ok = gr < nrow && gk + 8 <= kend;
                cp_async16(d, ok ? (const void*)(src + (long)gr * s_r + gk) : (const void*)src, ok);
            }
        }
    } else if (s_r == 1 && ((uintptr_t)src & 3) == 0 && (s_k & 1) == 0 && (row0 & 1) == 0) {
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
        const int ncm = groups * (UM_KC / 8);  // core matrices of the tile: (row group, K group)
        const int rl = 2 * (lane & 3), kl = lane >> 2;
        for (int c0 = warp * 32; c0 < ncm; c0 += nw * 32) {
            uint32_t w[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const int cm = c0 + j;
                const int kg = cm / groups, rg = cm - kg * groups;
                const int gr = row0 + rg * 8 + rl, gk = k0 + kg * 8 + kl;
                w[j] = 0u;
                if (cm < ncm && gk < kend && gr < nrow) {
                    const __nv_bfloat16* p = src + gr + (long)gk * s_k;
                    if (gr + 1 < nrow) w[j] = *reinterpret_cast<const uint32_t*>(p);
                    else w[j] = (uint32_t)__bfloat16_as_ushort(p[0]);
                }
            }
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const int cm = c0 + j;
                const uint32_t t = movmatrix_t(w[j]);  // every lane takes part (cm is warp-uniform)
                if (cm < ncm) *reinterpret_cast<uint32_t*>(dst + (cm << 7) + 4 * lane) = t;
            }
        }
    } else {
        for (int e = threadIdx.x; e < rows * UM_KC; e += blockDim.x) {
            int r, k;
            if (s_k == 1) { r = e / UM_KC; k = e - r * UM_KC; }  // lanes along the contiguous axis
            else { k = e / rows; r = e - k * rows; }
            put(r, k, get(r, k));
        }
    }
}

}  // namespace

// epi 0 store (split z writes Cf + z M N), 1 bias + GELU (Z -> Cf, gelu(Z) -> Hb), 2 dZ = acc gelu'(Zin) -> Hb
__global__ void __launch_bounds__(128, 1) k_umma_gemm(int M, int N, int K, const __nv_bfloat16* __restrict__ A, long sai,
                                                      long sak, const __nv_bfloat16* __restrict__ B, long sbk, long sbj,
                                                      int epi, float* __restrict__ Cf, const float* __restrict__ bias,
                                                      const float* __restrict__ Zin, __nv_bfloat16* __restrict__ Hb,
                                                      int kchunk, int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char um_smem[];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    const int Np = (N + 15) & ~15;                       // N of the MMA (multiple of 16)
    const uint32_t ncols = Np <= 32 ? 32u : (Np <= 64 ? 64u : (Np <= 128 ? 128u : 256u));
    const int a_bytes = UM_ROWS * UM_KC * 2, b_bytes = Np * UM_KC * 2;
    unsigned char* stA[2] = {um_smem, um_smem + a_bytes + b_bytes};
    unsigned char* stB[2] = {um_smem + a_bytes, um_smem + 2 * a_bytes + b_bytes};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i0 = blockIdx.y * UM_ROWS;
    const int kbeg = blockIdx.z * kchunk, kend = min(K, kbeg + kchunk);
    if (threadIdx.x == 0) { mbar_init(&s_bar[0]); mbar_init(&s_bar[1]); s_fail = 0; }
    if (warp == 0) {  // tensor memory for the accumulator: ncols FP32 columns x 128 lanes
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&s_tmem)), "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = umma_idesc(UM_ROWS, Np);
    const int nchunks = (kend - kbeg + UM_KC - 1) / UM_KC;
    int issued = 0;  // chunks whose MMAs were committed
    for (int c = 0; c < nchunks; ++c) {
        const int b = c & 1;
        if (c >= 2) {  // the stage's previous MMAs (chunk c - 2) must have read it
            if (threadIdx.x == 0 && !mbar_wait(&s_bar[b], (uint32_t)(((c >> 1) - 1) & 1))) s_fail = 1;
            __syncthreads();
            if (s_fail) break;
        }
        const int k0 = kbeg + c * UM_KC;
        stage_tile(stA[b], UM_ROWS, A, sai, sak, i0, M, k0, kend);
        stage_tile(stB[b], Np, B, sbj, sbk, 0, N, k0, kend);
        asm volatile("cp.async.wait_all;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic writes -> tensor-core reads
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = su32(stA[b]), b0 = su32(stB[b]);
#pragma unroll
            for (int s = 0; s < UM_KC / 16; ++s) {
                // K step s: core-matrix columns 2s and 2s + 1
                const uint64_t da = umma_sdesc(a0 + 2 * s * (UM_ROWS / 8) * 128, (UM_ROWS / 8) * 128, 128);
                const uint64_t db = umma_sdesc(b0 + 2 * s * (Np / 8) * 128, (Np / 8) * 128, 128);
                umma_issue(tmem, da, db, idesc, (c > 0 || s > 0) ? 1u : 0u);
            }
            umma_commit(&s_bar[b]);
        }
        issued = c + 1;
    }
    // completion of every MMA issued: the last commit's phase (bounded); after a failed
    // wait above, the chunks in flight are waited for the same way
    if (threadIdx.x == 0 && issued > 0) {
        const int cl = issued - 1;
        if (!mbar_wait(&s_bar[cl & 1], (uint32_t)((cl >> 1) & 1))) s_fail = 1;
        if (issued > 1 && s_fail) mbar_wait(&s_bar[(cl - 1) & 1], (uint32_t)(((cl - 1) >> 1) & 1));
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const bool ok = !s_fail;
    if (ok && nchunks > 0) {
        // each warp moves its 32 TMEM lanes (rows) through shared memory, 64 columns at a
        // time (32 x 65 floats per warp: the stages are free once every MMA has completed),
        // so that the epilogue's loads and stores run along the rows
        float* tile = reinterpret_cast<float*>(um_smem) + warp * (32 * 65);
        if (epi == 0) Cf += (size_t)blockIdx.z * M * N;
        for (int cb = 0; cb < Np; cb += 64) {
            const int cw = min(64, Np - cb);
            for (int c0 = 0; c0 < cw; c0 += 16) {
                uint32_t v[16];
                const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cb + c0);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                    "%13, %14, %15}, [%16];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int q = 0; q < 16; ++q) tile[lane * 65 + c0 + q] = __uint_as_float(v[q]);
            }
            __syncwarp();
            // eight rows at a time: their inputs (the tile, and Zin for the GELU gradient) are
            // loaded before any of them is computed and stored
            float bj[2] = {0.0f, 0.0f};
            if (epi == 1) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int jj = lane + 32 * h, j = cb + jj;
                    if (jj < cw && j < N) bj[h] = bias[j];
                }
            }
            for (int r0 = 0; r0 < 32; r0 += 8) {
                float av[8][2], zv[8][2];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int row = i0 + warp * 32 + r0 + u;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int jj = lane + 32 * h, j = cb + jj;
                        av[u][h] = tile[(r0 + u) * 65 + jj];
                        zv[u][h] = (epi == 2 && row < M && jj < cw && j < N) ? Zin[(long)row * N + j] : 0.0f;
                    }
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int row = i0 + warp * 32 + r0 + u;
                    if (row >= M) continue;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int jj = lane + 32 * h, j = cb + jj;
                        if (jj >= cw || j >= N) continue;
                        const float acc = av[u][h];
                        const long o = (long)row * N + j;
                        if (epi == 0) Cf[o] = acc;
                        else if (epi == 1) {
                            const float zz = acc + bj[h];
                            Cf[o] = zz;
                            Hb[o] = __float2bfloat16(gelu_dev(zz));
                        } else {
                            Hb[o] = __float2bfloat16(acc * gelu_grad_dev(zv[u][h]));
                        }
                    }
                }
            }
            __syncwarp();
        }
    } else if (!ok && threadIdx.x == 0 && err) {
        atomicExch(err, PHMC_ERR_BUDGET);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
}

// Shared memory of one launch: two stages of A (128 x 64) and B (Np x 64) BF16, at least the
// epilogue's four 32 x 65 float tiles.
static size_t umma_gemm_smem(int N) {
    const int Np = (N + 15) & ~15;
    const size_t stages = (size_t)2 * (UM_ROWS * UM_KC * 2 + Np * UM_KC * 2);
    const size_t epilogue = (size_t)4 * 32 * 65 * sizeof(float);  // the epilogue's row tiles (reuse the stages)
    return stages > epilogue ? stages : epilogue;
}

// A failed bounded wait of any launch on this device (PHMC_ERR_BUDGET), cleared when read.
static __device__ int g_umma_err;

// Launch: grid (1, ceil(M / 128), splits); each split covers kchunk of K.
cudaError_t launch_umma_gemm(int M, int N, int K, const __nv_bfloat16* A, long sai, long sak, const __nv_bfloat16* B,
                             long sbk, long sbj, int epi, float* Cf, const float* bias, const float* Zin,
                             __nv_bfloat16* Hb, int kchunk, int splits, cudaStream_t st) {
    if (N < 1 || N > 256) return cudaErrorInvalidValue;
    const size_t smem = umma_gemm_smem(N);
    cudaError_t e = cudaFuncSetAttribute(k_umma_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int* err = nullptr;
    e = cudaGetSymbolAddress((void**)&err, g_umma_err);
    if (e != cudaSuccess) return e;
    dim3 grid(1, (M + UM_ROWS - 1) / UM_ROWS, splits);
    k_umma_gemm<<<grid, 128, smem, st>>>(M, N, K, A, sai, sak, B, sbk, sbj, epi, Cf, bias, Zin, Hb, kchunk, err);
    return cudaGetLastError();
}

// The recorded error of this device's launches (0 none), cleared; synchronises the stream.
int umma_take_error(cudaStream_t st) {
    int v = 0;
    if (cudaStreamSynchronize(st) != cudaSuccess) return PHMC_ERR_CUDA;
    if (cudaMemcpyFromSymbol(&v, g_umma_err, sizeof(int)) != cudaSuccess) return PHMC_ERR_CUDA;
    if (v) {
        const int z = 0;
        if (cudaMemcpyToSymbol(g_umma_err, &z, sizeof(int)) != cudaSuccess) return PHMC_ERR_CUDA;
    }
    return v;
}
