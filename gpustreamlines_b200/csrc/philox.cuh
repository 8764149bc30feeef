// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
// "Parallel Random Numbers: As Easy as 1, 2, 3", SC'11), written for this
// library.  The stream layout follows curand_init(seed, subsequence, offset)
// as the reference calls it (generate_streamlines_cuda.cu:445,500,
// boot.cu:649,867, ptt_init.cu:28): the 64-bit seed is the key, a
// subsequence advances the high 64 bits of the 128-bit counter, the offset
// advances the low 64 bits in units of 4 outputs plus an index into the
// current 4-word block.  The layout and the uint->float mapping are pinned
// black-box against the CUDA toolkit's generator by the GPU test suite.
#pragma once
#include <cstdint>

namespace csl {

constexpr uint32_t kPhiloxM0 = 0xD2511F53u;
constexpr uint32_t kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u;
constexpr uint32_t kPhiloxW1 = 0xBB67AE85u;

__host__ __device__ __forceinline__ uint32_t mulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32);
#endif
}

__host__ __device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const uint32_t hi0 = mulhi32(kPhiloxM0, c.x);
        const uint32_t lo0 = kPhiloxM0 * c.x;
        const uint32_t hi1 = mulhi32(kPhiloxM1, c.z);
        const uint32_t lo1 = kPhiloxM1 * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += kPhiloxW0;
        k.y += kPhiloxW1;
    }
    return c;
}

// Generator state: 24 bytes of registers (curand's Philox state also caches
// Box-Muller values; this one keeps a separate normal cache only where used).
struct Philox {
    uint4 ctr;
    uint2 key;
    uint4 out;
    int idx;  // next word of `out` to return, 4 = exhausted

    __host__ __device__ __forceinline__ void init(uint64_t seed, uint64_t subsequence,
                                                  uint64_t offset) {
        key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
        ctr = make_uint4(0u, 0u, (uint32_t)subsequence, (uint32_t)(subsequence >> 32));
        const uint64_t blocks = offset >> 2;
        add_low(blocks);
        out = philox4x32_10(ctr, key);
        idx = (int)(offset & 3u);
    }

    // 128-bit counter += v
    __host__ __device__ __forceinline__ void add_low(uint64_t v) {
        const uint64_t lo = ((uint64_t)ctr.y << 32 | ctr.x);
        const uint64_t nlo = lo + v;
        ctr.x = (uint32_t)nlo;
        ctr.y = (uint32_t)(nlo >> 32);
        if (nlo < lo) {
            if (++ctr.z == 0u) ++ctr.w;
        }
    }

    __host__ __device__ __forceinline__ uint32_t next() {
        if (idx == 4) {
            add_low(1);
            out = philox4x32_10(ctr, key);
            idx = 0;
        }
        const int i = idx++;
        return i == 0 ? out.x : (i == 1 ? out.y : (i == 2 ? out.z : out.w));
    }

    // Uniform float in (0, 1]: u * 2^-32 + 2^-33 (the mid-point of each of the
    // 2^32 cells, rounded to float32).
    __host__ __device__ __forceinline__ float uniform() {
        return uint_to_uniform(next());
    }

    __host__ __device__ static __forceinline__ float uint_to_uniform(uint32_t x) {
        // one fused multiply-add, as the reference's fast-math build contracts it
        return fmaf((float)x, 2.3283064365386963e-10f, 2.3283064365386963e-10f / 2.0f);
    }
};

// Generator whose state lives in shared memory and is advanced by lane 0
// only (the probabilistic getter draws one uniform per step on lane 0).
struct PhiloxShared {
    Philox *st;
    __device__ __forceinline__ void init(uint64_t seed, uint64_t subsequence, uint64_t offset) {
        if ((threadIdx.x & 31) == 0) st->init(seed, subsequence, offset);
        __syncwarp();
    }
    __device__ __forceinline__ float uniform() { return st->uniform(); }
};

}  // namespace csl
