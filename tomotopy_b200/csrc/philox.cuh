// philox.cuh -- counter-based Philox4x32-10 (Salmon, Moraes, Dror & Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11), usable from host
// and device code.  Every random draw of the sampler is a pure function of
// (seed, counter), so results do not depend on thread scheduling.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define TMT_HD __host__ __device__ __forceinline__
#else
#define TMT_HD inline
#endif

namespace tmt {

// Stream tags: the third counter word of each use, so that the streams of
// initialisation, training sweeps, inference and corpus synthesis never overlap.
constexpr uint32_t kStreamInit = 0x494E4954u;   // 'INIT'
constexpr uint32_t kStreamSweep = 0x53574550u;  // 'SWEP'
constexpr uint32_t kStreamInfer = 0x494E4652u;  // 'INFR'
constexpr uint32_t kStreamSynth = 0x53594E54u;  // 'SYNT'

struct u32x4 { uint32_t x, y, z, w; };

TMT_HD void mulhilo(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo)
{
#if defined(__CUDA_ARCH__)
    lo = a * b;
    hi = __umulhi(a, b);
#else
    uint64_t p = (uint64_t)a * (uint64_t)b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
#endif
}

TMT_HD u32x4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo(0xD2511F53u, c0, hi0, lo0);
        mulhilo(0xCD9E8D57u, c2, hi1, lo1);
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return u32x4{ c0, c1, c2, c3 };
}

// First output word for counter (c0..c3) under a 64-bit key.
TMT_HD uint32_t philox_u32(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint64_t key)
{
    return philox4x32_10(c0, c1, c2, c3, (uint32_t)key, (uint32_t)(key >> 32)).x;
}

// Top 24 bits scaled to [0, 1): exact in float and strictly below 1.
TMT_HD float u01(uint32_t x)
{
    return (float)(x >> 8) * (1.0f / 16777216.0f);
}

} // namespace tmt
