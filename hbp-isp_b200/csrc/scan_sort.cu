// Device-wide exclusive scan and stable LSD radix sort (project kernels; the
// reference uses thrust::exclusive_scan / sort / sort_by_key at CRTrees.cu:395,
// segment.cu:1061-1064, hbp_isp.cu:888, :981, :993, :1012).
#include "engine.h"

namespace hbp
{
namespace
{
constexpr int ST = 256, SI = 8, STILE = ST * SI; // scan tile: 2048 ints

// Block-wide exclusive scan of one value per thread; returns the block total.
__device__ __forceinline__ int block_exscan(int v, int &total)
{
    __shared__ int wsum[ST / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1)
    {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o)
            x += y;
    }
    if (lane == 31)
        wsum[w] = x;
    __syncthreads();
    if (w == 0)
    {
        int s = lane < ST / 32 ? wsum[lane] : 0;
        for (int o = 1; o < 32; o <<= 1)
        {
            int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o)
                s += y;
        }
        if (lane < ST / 32)
            wsum[lane] = s;
    }
    __syncthreads();
    int base = w ? wsum[w - 1] : 0;
    total = wsum[ST / 32 - 1];
    __syncthreads();
    return base + x - v;
}

__global__ void __launch_bounds__(ST) scan_tiles(const int *__restrict__ in, int *__restrict__ out,
                                                 long n, int *__restrict__ tile_sums)
{
    const long t0 = (long)blockIdx.x * STILE + (long)threadIdx.x * SI;
    int v[SI];
    int s = 0;
#pragma unroll
    for (int k = 0; k < SI; ++k)
    {
        v[k] = t0 + k < n ? in[t0 + k] : 0;
        s += v[k];
    }
    int total;
    int ex = block_exscan(s, total);
#pragma unroll
    for (int k = 0; k < SI; ++k)
    {
        if (t0 + k < n)
            out[t0 + k] = ex;
        ex += v[k];
    }
    if (threadIdx.x == 0)
        tile_sums[blockIdx.x] = total;
}

__global__ void add_tile_offsets(int *__restrict__ out, long n, const int *__restrict__ offs)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        out[i] += offs[i / STILE];
}

__global__ void write_total(const int *in, const int *out, long n, int *total)
{
    *total = n > 0 ? out[n - 1] + in[n - 1] : 0;
}

void scan_rec(const int *in, int *out, long n, Arena &tmp, cudaStream_t st)
{
    long tiles = (n + STILE - 1) / STILE;
    int *sums = tmp.alloc<int>(tiles);
    scan_tiles<<<(int)tiles, ST, 0, st>>>(in, out, n, sums);
    note_launch();
    HBP_LAUNCH_CHECK();
    if (tiles > 1)
    {
        int *soff = tmp.alloc<int>(tiles);
        scan_rec(sums, soff, tiles, tmp, st);
        add_tile_offsets<<<ceil_div(n, 256), 256, 0, st>>>(out, n, soff);
        note_launch();
        HBP_LAUNCH_CHECK();
    }
}

// ---------------------------------------------------------------------------
// radix sort: tiles of 2048 items processed in 8 rounds of 256 consecutive
// items; per digit the offset of (digit, tile) comes from one exclusive scan
// over the digit-major histogram, the rank inside a tile follows input order.
constexpr int RT = 256, RI = 8, RTILE = RT * RI, RWARPS = RT / 32;

template <typename KT>
__global__ void __launch_bounds__(RT) radix_hist(const KT *__restrict__ keys, long n, int shift,
                                                 int *__restrict__ hist, int ntiles)
{
    __shared__ int h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const long base = (long)blockIdx.x * RTILE;
#pragma unroll
    for (int r = 0; r < RI; ++r)
    {
        long i = base + r * RT + threadIdx.x;
        if (i < n)
            atomicAdd(&h[(int)((keys[i] >> shift) & 255)], 1);
    }
    __syncthreads();
    hist[(long)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

template <typename KT, bool HAS_VAL>
__global__ void __launch_bounds__(RT)
    radix_scatter(const KT *__restrict__ keys, const uint32_t *__restrict__ vals, KT *__restrict__ okeys,
                  uint32_t *__restrict__ ovals, long n, int shift, const int *__restrict__ offs,
                  int ntiles)
{
    __shared__ int run[256];
    __shared__ int wcnt[RWARPS][256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    run[threadIdx.x] = offs[(long)threadIdx.x * ntiles + blockIdx.x];
    const long base = (long)blockIdx.x * RTILE;
    for (int r = 0; r < RI; ++r)
    {
#pragma unroll
        for (int k = 0; k < RWARPS; ++k)
            wcnt[k][threadIdx.x] = 0;
        __syncthreads();
        long i = base + r * RT + threadIdx.x;
        bool valid = i < n;
        KT key = valid ? keys[i] : (KT)0;
        int dg = valid ? (int)((key >> shift) & 255) : 256;
        unsigned peers = __match_any_sync(0xffffffffu, dg);
        int wrank = __popc(peers & lt);
        if (valid && wrank == 0)
            wcnt[w][dg] = __popc(peers);
        __syncthreads();
        if (valid)
        {
            int pos = run[dg] + wrank;
            for (int k = 0; k < w; ++k)
                pos += wcnt[k][dg];
            okeys[pos] = key;
            if (HAS_VAL)
                ovals[pos] = vals[i];
        }
        __syncthreads();
        int add = 0;
#pragma unroll
        for (int k = 0; k < RWARPS; ++k)
            add += wcnt[k][threadIdx.x];
        run[threadIdx.x] += add;
        __syncthreads();
    }
}

template <typename KT, bool HAS_VAL>
void radix_sort_impl(KT *keys, uint32_t *vals, KT *keys_alt, uint32_t *vals_alt, long n, int bits,
                     Arena &tmp, cudaStream_t st)
{
    if (n <= 1 || bits <= 0)
        return;
    const int ntiles = (int)((n + RTILE - 1) / RTILE);
    size_t m = tmp.mark();
    int *hist = tmp.alloc<int>((size_t)256 * ntiles);
    int *offs = tmp.alloc<int>((size_t)256 * ntiles);
    const int passes = (bits + 7) / 8;
    KT *ka = keys, *kb = keys_alt;
    uint32_t *va = vals, *vb = vals_alt;
    for (int p = 0; p < passes; ++p)
    {
        int shift = 8 * p;
        radix_hist<KT><<<ntiles, RT, 0, st>>>(ka, n, shift, hist, ntiles);
        note_launch();
        HBP_LAUNCH_CHECK();
        size_t m2 = tmp.mark();
        scan_rec(hist, offs, (long)256 * ntiles, tmp, st);
        tmp.rewind(m2);
        radix_scatter<KT, HAS_VAL><<<ntiles, RT, 0, st>>>(ka, va, kb, vb, n, shift, offs, ntiles);
        note_launch();
        HBP_LAUNCH_CHECK();
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    if (ka != keys)
    {
        HBP_CUDA(cudaMemcpyAsync(keys, ka, sizeof(KT) * n, cudaMemcpyDeviceToDevice, st));
        if (HAS_VAL)
            HBP_CUDA(cudaMemcpyAsync(vals, va, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
    }
    tmp.rewind(m);
}
} // namespace

void exclusive_scan(const int *in, int *out, long n, int *total_dev, Arena &tmp, cudaStream_t st)
{
    size_t m = tmp.mark();
    if (n > 0)
        scan_rec(in, out, n, tmp, st);
    if (total_dev)
    {
        write_total<<<1, 1, 0, st>>>(in, out, n, total_dev);
        note_launch();
        HBP_LAUNCH_CHECK();
    }
    tmp.rewind(m);
}

void radix_sort_pairs_u32(uint32_t *keys, uint32_t *vals, uint32_t *keys_alt, uint32_t *vals_alt,
                          long n, int bits, Arena &tmp, cudaStream_t st)
{
    radix_sort_impl<uint32_t, true>(keys, vals, keys_alt, vals_alt, n, bits, tmp, st);
}

void radix_sort_keys_u64(uint64_t *keys, uint64_t *keys_alt, long n, int bits, Arena &tmp,
                         cudaStream_t st)
{
    radix_sort_impl<uint64_t, false>(keys, nullptr, keys_alt, nullptr, n, bits, tmp, st);
}

} // namespace hbp
