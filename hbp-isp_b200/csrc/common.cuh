// Shared device/host helpers of the B200 HBP-ISP engine.
#pragma once

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

#include "hbp_b200.h"
#include <nvtx3/nvToolsExt.h>

namespace hbp
{

// ---------------------------------------------------------------------------
// error handling
struct CudaFailure
{
    cudaError_t err;
    const char *file;
    int line;
};

#define HBP_CUDA(x)                                                                                \
    do                                                                                             \
    {                                                                                              \
        cudaError_t e_ = (x);                                                                      \
        if (e_ != cudaSuccess)                                                                     \
            throw ::hbp::CudaFailure{e_, __FILE__, __LINE__};                                      \
    } while (0)

#define HBP_LAUNCH_CHECK() HBP_CUDA(cudaGetLastError())

struct StatusError
{
    hbp_status st;
    const char *what;
};

inline int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }

// Number of kernels this library has launched (reported by the benchmark).
extern std::atomic<long> g_launches;
inline void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// Device-side error word: kernels that give up a bounded wait or meet an
// impossible size record a code here instead of trapping; the host reads it.
enum DeviceErr : int
{
    DERR_NONE = 0,
    DERR_BARRIER_TIMEOUT = 1,
    DERR_NO_CONVERGENCE = 2,
    DERR_CAPACITY = 3,
};

// ---------------------------------------------------------------------------
// arithmetic shared with the CPU oracle (reference semantics)

// BSD LCG of hbp_isp.cu:551-559.
__host__ __device__ __forceinline__ uint32_t lcg(uint32_t s)
{
    return (1103515245u * s + 12345u) % 2147483648u;
}

// Grid-wide barrier for cooperative launches. Sense-reversing counter in
// global memory; every wait is bounded (spin_limit polls with nanosleep
// back-off) and, on time-out, the CTA records DERR_BARRIER_TIMEOUT and the
// caller stops work instead of hanging.
struct GridBarrier
{
    unsigned int *count; // [0] arrivals, [1] generation
    int *err;
};

constexpr long GRID_SPIN_LIMIT = 20000000; // ~ seconds with back-off

__device__ __forceinline__ bool grid_sync(GridBarrier b, unsigned int nblocks, long spin_limit = GRID_SPIN_LIMIT)
{
    __syncthreads();
    __shared__ int ok;
    if (threadIdx.x == 0)
    {
        ok = 1;
        volatile unsigned int *gen = b.count + 1;
        unsigned int g = *gen;
        __threadfence();
        unsigned int arrived = atomicAdd(b.count, 1u) + 1;
        if (arrived == nblocks)
        {
            atomicExch(b.count, 0u);
            __threadfence();
            atomicAdd(b.count + 1, 1u);
        }
        else
        {
            long spins = 0;
            while (*gen == g)
            {
                if (++spins > spin_limit || *(volatile int *)b.err == DERR_BARRIER_TIMEOUT)
                {
                    atomicExch(b.err, (int)DERR_BARRIER_TIMEOUT);
                    ok = 0;
                    break;
                }
                __nanosleep(spins < 1000 ? 32 : 256);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

__device__ __forceinline__ int warp_sum_int(int v)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// NVTX range for profilers (stage and pyramid level names); no cost when no
// tool is attached.
struct NvtxRange
{
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};

} // namespace hbp
