// Driver median (medianFilter of main_stereo_hbp_isp.cu:120-192) with its
// scratch in a file-scope device array instead of a context slab, for callers
// that may not allocate device memory (hbp_driver_median_noalloc_d).
#include <mutex>

#include "engine.h"

namespace hbp
{
namespace
{
// Scratch of the horizontal pass: HBP_NOALLOC_MAX_PIXELS floats (8 MiB). It is
// loaded with this file's module, i.e. on the first call on a device.
__device__ __align__(256) float g_median_scratch[HBP_NOALLOC_MAX_PIXELS];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
float *g_scratch_addr[MAX_DEVICES] = {};

__device__ __forceinline__ float median7_sorted(float *v)
{
    for (int j = 1; j < 7; ++j)
    {
        float t = v[j];
        int i = j - 1;
        while (i >= 0 && v[i] > t)
        {
            v[i + 1] = v[i];
            i--;
        }
        v[i + 1] = t;
    }
    return v[3];
}

// Horizontal pass writing EVERY scratch entry: 0 on the 3-pixel frame (the
// value the reference's zero-initialised temp keeps there, and the context
// path's cleared slab), the 7-tap median or the invalid disparity inside. The
// scratch therefore needs no clearing and keeps nothing from earlier calls.
__global__ void median_h_full_kernel(const float *D, int W, int H, float *T)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W * H)
        return;
    int y = i / W, u = i - y * W;
    if (u < 3 || u >= W - 3 || y < 3 || y >= H - 3)
    {
        T[i] = 0.0f;
        return;
    }
    if (D[i] >= 0)
    {
        float v[7];
        for (int k = 0; k < 7; ++k)
            v[k] = D[i - 3 + k];
        T[i] = median7_sorted(v);
    }
    else
        T[i] = D[i];
}

// Vertical pass: reads the scratch (including its zero frame rows) and writes
// the interior valid pixels of D.
__global__ void median_v_static_kernel(const float *T, int W, int H, float *D)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W * H)
        return;
    int y = i / W, u = i - y * W;
    if (u < 3 || u >= W - 3 || y < 3 || y >= H - 3)
        return;
    if (D[i] >= 0)
    {
        float v[7];
        for (int k = 0; k < 7; ++k)
            v[k] = T[(y - 3 + k) * W + u];
        D[i] = median7_sorted(v);
    }
}

// Device address of the scratch on the current device, looked up once per
// device (cudaGetSymbolAddress; the first lookup loads the module).
float *static_scratch()
{
    int dev = 0;
    HBP_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES)
        throw StatusError{HBP_ERR_INVALID_ARG, "device ordinal out of range for the static scratch table"};
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev])
    {
        void *p = nullptr;
        HBP_CUDA(cudaGetSymbolAddress(&p, g_median_scratch));
        g_scratch_addr[dev] = static_cast<float *>(p);
    }
    return g_scratch_addr[dev];
}
} // namespace

void launch_driver_median_noalloc(float *disp, int W, int H, cudaStream_t st)
{
    if (W <= 0 || H <= 0)
        throw StatusError{HBP_ERR_INVALID_ARG, "W and H must be positive"};
    const long n = (long)W * H;
    if (n > HBP_NOALLOC_MAX_PIXELS)
        throw StatusError{HBP_ERR_INVALID_ARG,
                          "W*H exceeds HBP_NOALLOC_MAX_PIXELS (2097152), the size of the static scratch"};
    float *T = static_scratch();
    median_h_full_kernel<<<ceil_div(n, 256), 256, 0, st>>>(disp, W, H, T);
    note_launch();
    median_v_static_kernel<<<ceil_div(n, 256), 256, 0, st>>>(T, W, H, disp);
    note_launch();
    HBP_LAUNCH_CHECK();
}

} // namespace hbp
