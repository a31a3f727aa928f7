// Force-included (nvcc -include) ahead of every reference source compiled into
// the checker library oracle/_ref/libhbpref.so. It changes no reference file;
// it only pins two behaviours that the reference leaves to chance:
//
//  1. Every cudaMalloc is padded by 64 KiB and zero-filled. The reference reads
//     a few elements past the end of the LAB image in compute_1nn_grid_k
//     (segment.cu:66 loads before the bounds test at :71) and never writes the
//     top pyramid level's planes before copying them as priors
//     (hbp_isp.cu:1333-1337 -> :68). Padding keeps the stray read inside the
//     allocation; zero-filling makes the first prior deterministic (all-zero
//     planes), which is what fresh device memory usually holds.
//
//  2. __float2int_rd keeps CUDA's own result for NaN (0) and for |x| < 2^30,
//     and clamps larger magnitudes to +-2^30. read_plane_cost (hbp_isp.cu:217-
//     223) computes d+1 after a saturating conversion; at +2^31-1 that wraps and
//     the volume index leaves the allocation. With the clamp such a plane reads
//     as out of range (cost = tau) instead of touching memory it does not own.
#pragma once
#include <cuda_runtime.h>

static inline cudaError_t hbp_ref_padded_malloc(void **p, size_t n)
{
    const size_t pad = 65536;
    cudaError_t e = ::cudaMalloc(p, n + pad);
    if (e == cudaSuccess)
        e = ::cudaMemset(*p, 0, n + pad);
    return e;
}
template <typename T>
static inline cudaError_t hbp_ref_padded_malloc_t(T **p, size_t n)
{
    return hbp_ref_padded_malloc((void **)p, n);
}

#ifdef __CUDACC__
static __device__ __forceinline__ int hbp_ref_f2i_rd(float x)
{
    if (x != x)
        return __float2int_rd(x);
    const float lim = 1073741824.0f; // 2^30
    x = x > lim ? lim : (x < -lim ? -lim : x);
    return __float2int_rd(x);
}
#define __float2int_rd(x) hbp_ref_f2i_rd(x)
#endif

#define cudaMalloc hbp_ref_padded_malloc_t
