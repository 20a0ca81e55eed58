// Surrogate network: constants of the move descriptor, the device view of an
// attached network and the BF16 tensor-core forward pass shared by the
// standalone GEMM path (k_mlp.cu) and the in-kernel first stage (k_mc.cu).
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#define SUR_SHELLS 16      // radial shells of width 0.5 sigma out to 8 sigma
#define SUR_CLASSES 4      // +1 (charged site, cation), -1, neutral titratable site, permanent +1
#define SUR_RMAX 8.0f
#define SUR_K 80           // network input width (71 used, zero padded to a multiple of 16)
#define SUR_USED 71
#define SUR_ROWS 4         // rows per move: old / new state of <= 2 changed particles
#define SUR_AST 136        // shared-memory activation row stride (bf16 elements)
#define SUR_HMAX 128

// feature layout of one row
//   [0, 64)  shell s, class c at s * 4 + c: particles of the environment (the
//            changed particles excluded) with s = floor(2 r)
//   64       z / (slab height)
//   65..68   one-hot state of the row's particle: charged site, neutral site, anion, cation
//   69       pKa - pH
//   70       log10(reservoir salt concentration), -10 when there is none

// Device view of the network attached to an engine (H == 0: none).
struct SurDev {
    const uint2* w[3];        // hidden layers, fragment-packed BF16 (see sur_pack_index)
    const float* b[3];        // hidden biases (FP32)
    const uint16_t* w4;       // output weights (BF16 bits)
    const float* b4;          // output bias
    const float* mu;          // input standardisation
    const float* sd;
    float scale, offset;      // energy = y * scale + offset
    int H;
};

// Fragment-packed layout of a K x H weight matrix for mma.sync m16n8k16: column
// group cg (16 outputs), k-step ks, n-tile nt, lane -> one uint2 holding the
// lane's two B registers.
__host__ __device__ inline size_t sur_pack_index(int cg, int ks, int nt, int lane, int nks) {
    return (((size_t)cg * nks + ks) * 2 + nt) * 32 + lane;
}

__device__ __forceinline__ float sur_gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752440f)); }

__device__ __forceinline__ void sur_mma(float* c, const uint32_t* a, uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Output layer of one row (one warp): sum_k h[k] w4[k] in a fixed lane order.
__device__ __forceinline__ float sur_out_dot(const __nv_bfloat16* h, const uint16_t* w4, int H, int lane) {
    float v = 0.0f;
    for (int k = lane; k < H; k += 32)
        v += __bfloat162float(h[k]) * __bfloat162float(__ushort_as_bfloat16(w4[k]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ---- bulk asynchronous copies (global -> this block's shared memory) ----
__device__ __forceinline__ void sur_mbar_init(uint64_t* mbar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// One thread: order earlier generic accesses of the block (made visible by a
// preceding __syncthreads) before the async copy, then copy `bytes` (multiple
// of 16, both addresses 16-byte aligned) and count them on `mbar`.
__device__ __forceinline__ void sur_bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* mbar) {
    const uint32_t m = (uint32_t)__cvta_generic_to_shared(mbar);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(m), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src), "r"(bytes), "r"(m)
                 : "memory");
}
// Bounded wait for the completion of the phase with parity `parity`; false when the bound ran out.
__device__ __forceinline__ bool sur_mbar_wait(uint64_t* mbar, uint32_t parity) {
    const uint32_t m = (uint32_t)__cvta_generic_to_shared(mbar);
    for (int it = 0; it < (1 << 20); ++it) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(m), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}
__host__ __device__ inline uint32_t sur_layer_bytes(int K, int H) { return (uint32_t)K * (uint32_t)H * 2u; }

// Shared-memory layout of the staged first stage: two 16-row activation
// buffers, then the three hidden layers' weights (SUR_K x SUR_HMAX, then two
// SUR_HMAX x SUR_HMAX, BF16, fragment-packed).
#define SUR_ACT_BYTES (2 * 16 * SUR_AST * 2)
#define SUR_WBUF_BYTES (SUR_HMAX * SUR_HMAX * 2)
#define SUR_SMEM_BYTES (128 + SUR_ACT_BYTES + SUR_K * SUR_HMAX * 2 + 2 * SUR_WBUF_BYTES)
// two-buffer layout: layer 3 streams into layer 1's buffer once layer 1 is done
#define SUR_SMEM2_BYTES (128 + SUR_ACT_BYTES + 2 * SUR_WBUF_BYTES)

// The caller's thread 0 has issued layer l -> w_l on mbar[l] (l = 0, 1, and 2
// unless late_l3), each barrier in the phase of parity `par`; with late_l3 layer 3
// is copied into wc (= wa) here, once layer 1 is done.  Computes the outputs
// (energy units) of rows 0..nrows-1 (nrows <= 8) held, standardised, in buf0.
// Returns false (every thread) when a copy did not arrive within the bound.
template <int NT>
__device__ bool sur_forward_staged(const SurDev& s, int nrows, __nv_bfloat16* buf0, __nv_bfloat16* buf1, const uint2* wa,
                                   const uint2* wb, const uint2* wc, uint64_t* mbar, uint32_t par, float* out, int* s_fail,
                                   bool late_l3, const uint16_t* w4) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t4 = lane & 3;
    __nv_bfloat16* in = buf0;
    __nv_bfloat16* ot = buf1;
    int K = SUR_K;
    for (int l = 0; l < 3; ++l) {
        const uint2* w = (l == 0) ? wa : (l == 1 ? wb : wc);
        bool ok = sur_mbar_wait(&mbar[l], par);
        if (!ok) ok = sur_mbar_wait(&mbar[l], par);  // a second bounded wait for the copy in flight
        if (!ok) *s_fail = 1;
        const int nks = K >> 4;
        for (int cg = warp; cg < (s.H >> 4); cg += NT / 32) {
            // even and odd k-steps accumulate separately (two independent MMA chains per n-tile)
            float acc[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
            float acc2[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
#pragma unroll 4
            for (int ks = 0; ks < nks; ++ks) {
                const __nv_bfloat16* p0 = in + g * SUR_AST + ks * 16 + 2 * t4;
                uint32_t a[4];
                a[0] = *reinterpret_cast<const uint32_t*>(p0);
                a[1] = *reinterpret_cast<const uint32_t*>(p0 + 8 * SUR_AST);
                a[2] = *reinterpret_cast<const uint32_t*>(p0 + 8);
                a[3] = *reinterpret_cast<const uint32_t*>(p0 + 8 * SUR_AST + 8);
                const uint2* wp = w + sur_pack_index(cg, ks, 0, lane, nks);
                const uint2 b0 = wp[0], b1 = wp[32];
                if (ks & 1) {
                    sur_mma(acc2[0], a, b0.x, b0.y);
                    sur_mma(acc2[1], a, b1.x, b1.y);
                } else {
                    sur_mma(acc[0], a, b0.x, b0.y);
                    sur_mma(acc[1], a, b1.x, b1.y);
                }
            }
#pragma unroll
            for (int nt = 0; nt < 2; ++nt)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[nt][q] += acc2[nt][q];
            if (g < nrows) {
#pragma unroll
                for (int nt = 0; nt < 2; ++nt)
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        const int col = cg * 16 + nt * 8 + 2 * t4 + q;
                        const float z = acc[nt][q] + __ldg(&s.b[l][col]);
                        ot[g * SUR_AST + col] = __float2bfloat16(sur_gelu(z));
                    }
            }
        }
        __syncthreads();
        if (l == 0 && late_l3 && threadIdx.x == 0)
            sur_bulk_load(const_cast<uint2*>(wc), s.w[2], sur_layer_bytes(s.H, s.H), &mbar[2]);
        __nv_bfloat16* t = in; in = ot; ot = t;
        K = s.H;
    }
    if (warp < nrows) {
        const float v = sur_out_dot(in + warp * SUR_AST, w4, s.H, lane);
        if (lane == 0) out[warp] = __fmaf_rn(v + __ldg(s.b4), s.scale, s.offset);
    }
    __syncthreads();
    return *s_fail == 0;
}
