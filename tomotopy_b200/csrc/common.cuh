// common.cuh -- small device helpers and host error types shared by the
// engine's translation units.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <stdexcept>
#include <string>

namespace tmtk {

constexpr unsigned FULL = 0xFFFFFFFFu;

__device__ __forceinline__ float hs_scan32(float x, int lane)
{
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const float y = __shfl_up_sync(FULL, x, off);
        if (lane >= off) x = __fadd_rn(x, y);
    }
    return x;
}

// the first `steps` steps of hs_scan32 (steps is warp-uniform, 0..5)
__device__ __forceinline__ float hs_scan_n(float x, int lane, int steps)
{
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        if (i < steps) {
            const float y = __shfl_up_sync(FULL, x, 1 << i);
            if (lane >= (1 << i)) x = __fadd_rn(x, y);
        }
    }
    return x;
}

__host__ __device__ __forceinline__ uint32_t round4(uint32_t x) { return (x + 3u) & ~3u; }

__device__ __forceinline__ double warp_sum(double x)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(FULL, x, o);
    return x;
}

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct ArgError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct OomError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct StateError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            throw CudaError(std::string(#call) + ": " + cudaGetErrorString(e_));              \
    } while (0)


} // namespace tmtk
