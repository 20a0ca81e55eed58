// The reference driver's random stream, restated for the device: a 32-bit
// Mersenne Twister (MT19937, Matsumoto & Nishimura, ACM TOMACS 8 (1998) 3-30)
// and the two draws the reference's move loops take from it
// (MC/src/mc.cu:62-65 choose_one, and uniform_real_distribution<real>(0, 1) at
// MC/src/mc.cu:204,353-354), with the arithmetic of GCC 13's libstdc++:
//   * uniform integer in [0, n): Lemire's multiply-and-reject reduction
//     ("Fast random integer generation in an interval", ACM TOMACS 29 (2019) 3:1-3:12)
//     of one 32-bit output to 64 bits; a rejection draws again;
//   * uniform float in [0, 1): one 32-bit output converted to float (round to
//     nearest) and scaled by 2^-32; a result that rounds up to 1 becomes the largest
//     float below 1.
// The state is the generator's 624 words and its position in them, in the order
// std::mt19937's stream output writes them, so a host generator hands its stream
// to the device and takes it back where the device left it.
#pragma once
#include <cstdint>

#ifndef __CUDACC__
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#endif

#define MT_N 624
#define MT_M 397

struct MtState {
    uint32_t x[MT_N];
    int p;  // next word to temper; MT_N: regenerate first
};

__host__ __device__ inline void mt_regenerate(MtState& s) {
    for (int i = 0; i < MT_N; ++i) {
        const uint32_t y = (s.x[i] & 0x80000000u) | (s.x[i + 1 < MT_N ? i + 1 : i + 1 - MT_N] & 0x7fffffffu);
        const int k = i + MT_M < MT_N ? i + MT_M : i + MT_M - MT_N;
        s.x[i] = s.x[k] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
    }
    s.p = 0;
}

__host__ __device__ inline uint32_t mt_next(MtState& s) {
    if (s.p >= MT_N) mt_regenerate(s);
    uint32_t y = s.x[s.p++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

// seeding of a default-constructed or integer-seeded generator (Knuth's multiplier 1812433253)
__host__ __device__ inline void mt_seed(MtState& s, uint32_t seed) {
    s.x[0] = seed;
    for (int i = 1; i < MT_N; ++i) s.x[i] = 1812433253u * (s.x[i - 1] ^ (s.x[i - 1] >> 30)) + (uint32_t)i;
    s.p = MT_N;
}

// uniform integer in [0, n), n >= 1 (one draw, more on rejection; n == 1 still draws once)
__host__ __device__ inline int mt_index(MtState& s, uint32_t n) {
    uint64_t prod = (uint64_t)mt_next(s) * (uint64_t)n;
    uint32_t low = (uint32_t)prod;
    if (low < n) {
        const uint32_t threshold = (uint32_t)(0u - n) % n;
        while (low < threshold) {
            prod = (uint64_t)mt_next(s) * (uint64_t)n;
            low = (uint32_t)prod;
        }
    }
    return (int)(prod >> 32);
}

// uniform float in [0, 1) (one draw)
__host__ __device__ inline float mt_unit_float(MtState& s) {
    const float v = (float)mt_next(s) * 2.3283064365386963e-10f;  // 2^-32: exact scaling
    return v >= 1.0f ? 0.99999994f : v;                            // largest float below 1
}
