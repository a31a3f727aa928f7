// Post-processing: left-right check with nearest-neighbour plane fill,
// colour-weighted median over planes, plane -> disparity, and the single-pair
// driver's 7-tap separable median. Reference: PostProcess (post_process.cu:
// 4-185, :373-390; CPU/OpenMP there) and medianFilter
// (main_stereo_hbp_isp.cu:120-192).
#include <cfloat>
#include <cmath>

#include "engine.h"

namespace hbp
{
namespace
{
__device__ __forceinline__ float get_z(const float *v, int x, int y)
{
    return v[0] * (float)x + v[1] * (float)y + v[2];
}

// doConsistencyCheck (post_process.cu:4-41), left view: fail where the right
// disparity at int(x - d + 0.5f) differs by more than 1.5.
__global__ void lr_fail_kernel(const float *dispL, const float *dispR, int W, int H, uint8_t *fail)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W * H)
        return;
    int y = i / W, x = i - y * W;
    float ds = dispL[i];
    uint8_t f = 0;
    if (ds == ds)
    {
        int rx = (int)((float)x - ds * 1.0f + 0.5f);
        if (rx >= 0 && rx < W && fabsf(dispR[y * W + rx] - ds) > 1.5f)
            f = 255;
    }
    fail[i] = f;
}

// cv::dilate with a 3x3 box; samples outside the image do not take part.
__global__ void dilate3_kernel(const uint8_t *in, int W, int H, uint8_t *out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W * H)
        return;
    int y = i / W, x = i - y * W;
    uint8_t m = 0;
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx)
        {
            int yy = y + dy, xx = x + dx;
            if (yy >= 0 && yy < H && xx >= 0 && xx < W)
                m = max(m, in[yy * W + xx]);
        }
    out[i] = m;
}

// Horizontal NN-interpolation (post_process.cu:72-109): nearest pixel on
// each side outside the dilated mask; keep the plane with the smaller
// disparity at the failed pixel. Reads only pixels outside the dilated mask,
// writes only failed pixels (a subset of it), so the update is in place.
__global__ void lr_fill_kernel(const uint8_t *fail, const uint8_t *fail2, int W, int H, float *plane)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W * H || !fail[i])
        return;
    int y = i / W, x = i - y * W;
    int xl = x, xr = x;
    while (xl >= 0 && fail2[y * W + xl] == 255)
        xl--;
    while (xr < W && fail2[y * W + xr] == 255)
        xr++;
    const float *pl = xl >= 0 ? plane + 3 * (size_t)(y * W + xl) : nullptr;
    const float *pr = xr < W ? plane + 3 * (size_t)(y * W + xr) : nullptr;
    const float *pick;
    if (!pl && !pr)
        return;
    else if (!pl)
        pick = pr;
    else if (!pr)
        pick = pl;
    else
        pick = get_z(pl, x, y) < get_z(pr, x, y) ? pl : pr;
    float a = pick[0], b = pick[1], c = pick[2];
    plane[3 * (size_t)i] = a;
    plane[3 * (size_t)i + 1] = b;
    plane[3 * (size_t)i + 2] = c;
}

__global__ void plane_to_disp_kernel(const float *plane, int W, int H, float *disp)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W * H)
        return;
    int y = i / W, x = i - y * W;
    disp[i] = get_z(plane + 3 * (size_t)i, x, y);
}

__global__ void compact_fail(const uint8_t *fail, int n, int *list, int *count)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && fail[i])
        list[atomicAdd(count, 1)] = i;
}

// Weighted median (post_process.cu:127-185): one block per failed pixel.
// Window samples (41x41 clipped) get weight expf(-sum|dBGR| / 10) and the
// disparity of their plane at the pixel; the samples are sorted by
// (disparity, window position) and the first one whose cumulative weight
// exceeds half the total gives the plane. Weight sums are in double.
// The colour distance sum|dBGR| is an integer 0..765, so the weights come
// from a 766-entry table computed on the host with the C library's expf,
// the function the reference's CPU code calls.
constexpr int WM_T = 256, WM_N = 2048, WM_R = 20;
__global__ void __launch_bounds__(WM_T)
    weighted_median_kernel(const uint8_t *bgr, const int *list, int W, int H, const float *plane_in,
                           float *plane_out, const float *wtab)
{
    __shared__ float zk[WM_N];
    __shared__ int ik[WM_N];
    __shared__ double part[WM_T];
    __shared__ int found;
    const int p = list[blockIdx.x];
    const int y = p / W, x = p - y * W;
    const int y0 = max(y - WM_R, 0), y1 = min(y + WM_R + 1, H);
    const int x0 = max(x - WM_R, 0), x1 = min(x + WM_R + 1, W);
    const int ww = x1 - x0, n = ww * (y1 - y0);
    const uint8_t *s = bgr + 3 * (size_t)p;
    const float s0 = s[0], s1 = s[1], s2 = s[2];
    for (int j = threadIdx.x; j < WM_N; j += WM_T)
    {
        if (j < n)
        {
            int q = (y0 + j / ww) * W + x0 + j % ww;
            zk[j] = get_z(plane_in + 3 * (size_t)q, x, y);
            ik[j] = j;
        }
        else
        {
            zk[j] = FLT_MAX;
            ik[j] = WM_N + j;
        }
    }
    __syncthreads();
    // bitonic sort by (z, index)
    for (int k = 2; k <= WM_N; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1)
        {
            for (int t = threadIdx.x; t < WM_N; t += WM_T)
            {
                int u = t ^ j;
                if (u > t)
                {
                    bool up = (t & k) == 0;
                    float za = zk[t], zb = zk[u];
                    int ia = ik[t], ib = ik[u];
                    bool gt = za > zb || (za == zb && ia > ib);
                    if (gt == up)
                    {
                        zk[t] = zb;
                        zk[u] = za;
                        ik[t] = ib;
                        ik[u] = ia;
                    }
                }
            }
            __syncthreads();
        }
    // weights in sorted order; block prefix sums in double (fixed order)
    const int per = WM_N / WM_T; // 8 consecutive sorted samples per thread
    double wv[per];
    double tsum = 0.0;
    for (int k = 0; k < per; ++k)
    {
        int j = threadIdx.x * per + k;
        double w = 0.0;
        if (j < n)
        {
            int src = ik[j];
            int q = (y0 + src / ww) * W + x0 + src % ww;
            const uint8_t *t = bgr + 3 * (size_t)q;
            int absdiff = abs((int)s0 - (int)t[0]) + abs((int)s1 - (int)t[1]) + abs((int)s2 - (int)t[2]);
            w = (double)wtab[absdiff];
        }
        wv[k] = w;
        tsum += w;
    }
    part[threadIdx.x] = tsum;
    if (threadIdx.x == 0)
        found = 0x7fffffff;
    __syncthreads();
    // inclusive scan of per-thread sums (Hillis-Steele, fixed order)
    for (int off = 1; off < WM_T; off <<= 1)
    {
        double v = threadIdx.x >= off ? part[threadIdx.x - off] : 0.0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    const double center = part[WM_T - 1] / 2.0;
    double run = threadIdx.x ? part[threadIdx.x - 1] : 0.0;
    for (int k = 0; k < per; ++k)
    {
        int j = threadIdx.x * per + k;
        run += wv[k];
        if (j < n && run > center)
        {
            atomicMin(&found, j);
            break;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && found < n)
    {
        int src = ik[found];
        int q = (y0 + src / ww) * W + x0 + src % ww;
        plane_out[3 * (size_t)p] = plane_in[3 * (size_t)q];
        plane_out[3 * (size_t)p + 1] = plane_in[3 * (size_t)q + 1];
        plane_out[3 * (size_t)p + 2] = plane_in[3 * (size_t)q + 2];
    }
}

// PostProcess::median_filter_gpu (post_process.cu:188-371), the reference's
// GPU variant of the weighted median: one warp per failed pixel. Window
// samples in row-major order get the device patch weight wtab[sum|dBGR|]
// (expf(-k / 10), launch_patch_weights) and z = fma(a, x, b * y) + c, the
// reference device code's evaluation of a * x + b * y + c; the total weight
// is a float sum in window order. The reference orders the samples with
// bubble_sort (:216-229): step i swaps into position i, in scan order, every
// later sample smaller than the current one there. Its effect is a rotation
// along the chain of strict running minima of [i, n): position i takes the
// last of the chain, each chain member the previous one's sample, the first
// member the old sample at i; position i is then final. Each step cuts
// [i+1, n) into 32 contiguous chunks (an odd chunk length keeps the lanes in
// distinct shared-memory banks), finds the running minimum before each chunk
// by an ordered scan of the chunk minima, reads the samples the chain hands
// on across chunk borders, then lets each lane walk its chunk carrying the
// previous chain member's sample. The running weight in float stops the sort
// at the first sample past half the total, whose plane is taken. NaN
// disparities never enter a chain, as NaN compares false there.
constexpr int WG_MAXN = (2 * WM_R + 1) * (2 * WM_R + 1); // window samples (1681)
constexpr int WG_W = 2;                                    // pixels (warps) per block

// the earlier of two (z, pos) candidates unless the later is strictly smaller;
// pos < 0: none
__device__ __forceinline__ void first_min(float &z, int &p, float z2, int p2)
{
    if (p2 >= 0 && (p < 0 || z2 < z))
    {
        z = z2;
        p = p2;
    }
}

__global__ void __launch_bounds__(32 * WG_W)
    weighted_median_gpu_kernel(const uint8_t *__restrict__ bgr, const int *__restrict__ list, int nf, int W,
                               int H, const float *__restrict__ plane_in, float *__restrict__ plane_out,
                               const float *__restrict__ wtab)
{
    __shared__ float zs_all[WG_W][WG_MAXN], ws_all[WG_W][WG_MAXN];
    __shared__ int ids_all[WG_W][WG_MAXN];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int item = blockIdx.x * WG_W + wid;
    if (item >= nf) // warp-uniform
        return;
    float *zs = zs_all[wid], *ws = ws_all[wid];
    int *ids = ids_all[wid];
    const int p = list[item];
    const int y = p / W, x = p - y * W;
    const int y0 = max(y - WM_R, 0), y1 = min(y + WM_R, H - 1);
    const int x0 = max(x - WM_R, 0), x1 = min(x + WM_R, W - 1);
    const int ww = x1 - x0 + 1, n = ww * (y1 - y0 + 1);
    const uint8_t *s = bgr + 3 * (size_t)p;
    const float fx = (float)x, fy = (float)y;
    for (int j = lane; j < n; j += 32)
    {
        const int q = (y0 + j / ww) * W + x0 + j % ww;
        const uint8_t *t = bgr + 3 * (size_t)q;
        const int d = abs((int)s[0] - (int)t[0]) + abs((int)s[1] - (int)t[1]) + abs((int)s[2] - (int)t[2]);
        ws[j] = wtab[d];
        const float *pl = plane_in + 3 * (size_t)q;
        zs[j] = __fadd_rn(__fmaf_rn(pl[0], fx, __fmul_rn(pl[1], fy)), pl[2]);
        ids[j] = j;
    }
    __syncwarp();
    float center = 0.f;
    if (lane == 0)
    {
        float sum = 0.f;
        for (int j = 0; j < n; ++j)
            sum = __fadd_rn(sum, ws[j]);
        center = __fdiv_rn(sum, 2.0f);
    }
    float run = 0.f; // lane 0's running weight in sorted order
    int pick = -1;
    for (int i = 0; i < n; ++i)
    {
        const float zi = zs[i];
        const bool chain = zi == zi; // a NaN at i is never displaced
        const int m = n - i - 1;
        const int c = ((m + 31) >> 5) | 1;
        const int lo = min(i + 1 + lane * c, n), hi = min(lo + c, n);
        // the chunk's first minimum (NaN samples never qualify)
        float cz = 0.f;
        int cp = -1;
        for (int j = lo; j < hi; ++j)
        {
            const float zj = zs[j];
            if (zj == zj)
                first_min(cz, cp, zj, j);
        }
        // ordered inclusive scan of the chunk minima over the lanes
        float sz = cz;
        int sp = cp;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1)
        {
            const float oz = __shfl_up_sync(0xffffffffu, sz, off);
            const int op = __shfl_up_sync(0xffffffffu, sp, off);
            if (lane >= off)
            {
                float nz = oz;
                int np = op;
                first_min(nz, np, sz, sp);
                sz = nz;
                sp = np;
            }
        }
        float pz = zi; // the running minimum before this lane's chunk
        int pp = i;
        {
            const float ez = __shfl_up_sync(0xffffffffu, sz, 1);
            const int ep = __shfl_up_sync(0xffffffffu, sp, 1);
            if (lane > 0)
                first_min(pz, pp, ez, ep);
        }
        float tz = zi; // the chain's end over the whole range
        int tpos = i;
        first_min(tz, tpos, __shfl_sync(0xffffffffu, sz, 31), __shfl_sync(0xffffffffu, sp, 31));
        // the samples handed on: the running minimum before the chunk, the
        // chain's end (to position i) and the sample at i
        float hz = zs[pp], hw = ws[pp];
        int hi_ = ids[pp];
        const float end_z = zs[tpos], end_w = ws[tpos];
        const int end_i = ids[tpos];
        const float wi = ws[i];
        const int ii = ids[i];
        __syncwarp();
        if (chain)
        {
            float curz = pz;
            for (int j = lo; j < hi; ++j)
            {
                const float zj = zs[j];
                if (zj < curz)
                {
                    const float wj = ws[j];
                    const int ij = ids[j];
                    zs[j] = hz;
                    ws[j] = hw;
                    ids[j] = hi_;
                    hz = zj;
                    hw = wj;
                    hi_ = ij;
                    curz = zj;
                }
            }
        }
        const bool moved = chain && tpos != i;
        if (lane == 0)
        {
            if (moved)
            {
                zs[i] = end_z;
                ws[i] = end_w;
                ids[i] = end_i;
            }
            run = __fadd_rn(run, moved ? end_w : wi);
            if (run > center)
                pick = moved ? end_i : ii;
        }
        pick = __shfl_sync(0xffffffffu, pick, 0);
        __syncwarp();
        if (pick >= 0)
            break;
    }
    if (lane == 0 && pick >= 0)
    {
        const int q = (y0 + pick / ww) * W + x0 + pick % ww;
        plane_out[3 * (size_t)p] = plane_in[3 * (size_t)q];
        plane_out[3 * (size_t)p + 1] = plane_in[3 * (size_t)q + 1];
        plane_out[3 * (size_t)p + 2] = plane_in[3 * (size_t)q + 2];
    }
}

__device__ __forceinline__ float median7(float *v)
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

// medianFilter, horizontal pass: interior pixels of D into T (T starts zero).
__global__ void median_h_kernel(const float *D, int W, int H, float *T)
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
            v[k] = D[i - 3 + k];
        T[i] = median7(v);
    }
    else
        T[i] = D[i];
}

// vertical pass: reads T (including its untouched zero border rows).
__global__ void median_v_kernel(const float *T, int W, int H, float *D)
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
        D[i] = median7(v);
    }
}
} // namespace

void launch_lr_check(const float *dispL, const float *dispR, float *planeL, uint8_t *fail,
                     uint8_t *fail2, int W, int H, cudaStream_t st)
{
    int n = W * H;
    lr_fail_kernel<<<ceil_div(n, 256), 256, 0, st>>>(dispL, dispR, W, H, fail);
    note_launch();
    dilate3_kernel<<<ceil_div(n, 256), 256, 0, st>>>(fail, W, H, fail2);
    note_launch();
    lr_fill_kernel<<<ceil_div(n, 256), 256, 0, st>>>(fail, fail2, W, H, planeL);
    note_launch();
    HBP_LAUNCH_CHECK();
}

void launch_plane_to_disp(const float *plane, float *disp, int W, int H, cudaStream_t st)
{
    plane_to_disp_kernel<<<ceil_div(W * H, 256), 256, 0, st>>>(plane, W, H, disp);
    note_launch();
    HBP_LAUNCH_CHECK();
}

void launch_weighted_median_gpu(const uint8_t *bgr, const uint8_t *fail, const float *plane_in,
                                float *plane_out, int W, int H, const float *wtab766, Arena &tmp,
                                cudaStream_t st)
{
    int n = W * H;
    size_t m = tmp.mark();
    int *list = tmp.alloc<int>(n), *count = tmp.alloc<int>(1);
    HBP_CUDA(cudaMemsetAsync(count, 0, sizeof(int), st));
    HBP_CUDA(cudaMemcpyAsync(plane_out, plane_in, sizeof(float) * 3 * (size_t)n, cudaMemcpyDeviceToDevice, st));
    compact_fail<<<ceil_div(n, 256), 256, 0, st>>>(fail, n, list, count);
    note_launch();
    HBP_LAUNCH_CHECK();
    int nf = 0;
    HBP_CUDA(cudaMemcpyAsync(&nf, count, sizeof(int), cudaMemcpyDeviceToHost, st));
    HBP_CUDA(cudaStreamSynchronize(st));
    if (nf > 0)
    {
        weighted_median_gpu_kernel<<<ceil_div(nf, WG_W), 32 * WG_W, 0, st>>>(bgr, list, nf, W, H, plane_in,
                                                                               plane_out, wtab766);
        note_launch();
        HBP_LAUNCH_CHECK();
    }
    tmp.rewind(m);
}

void median_weight_table(float *host766)
{
    for (int k = 0; k < 766; ++k)
        host766[k] = std::exp(-(float)k / 10.0f);
}

void launch_weighted_median(const uint8_t *bgr, const uint8_t *fail, const float *plane_in,
                            float *plane_out, int W, int H, const float *wtab, Arena &tmp,
                            cudaStream_t st)
{
    int n = W * H;
    size_t m = tmp.mark();
    int *list = tmp.alloc<int>(n), *count = tmp.alloc<int>(1);
    HBP_CUDA(cudaMemsetAsync(count, 0, sizeof(int), st));
    HBP_CUDA(cudaMemcpyAsync(plane_out, plane_in, sizeof(float) * 3 * (size_t)n, cudaMemcpyDeviceToDevice, st));
    compact_fail<<<ceil_div(n, 256), 256, 0, st>>>(fail, n, list, count);
    note_launch();
    HBP_LAUNCH_CHECK();
    int nf = 0;
    HBP_CUDA(cudaMemcpyAsync(&nf, count, sizeof(int), cudaMemcpyDeviceToHost, st));
    HBP_CUDA(cudaStreamSynchronize(st));
    if (nf > 0)
    {
        weighted_median_kernel<<<nf, WM_T, 0, st>>>(bgr, list, W, H, plane_in, plane_out, wtab);
        note_launch();
        HBP_LAUNCH_CHECK();
    }
    tmp.rewind(m);
}

void launch_driver_median(float *disp, float *tmp, int W, int H, cudaStream_t st)
{
    int n = W * H;
    HBP_CUDA(cudaMemsetAsync(tmp, 0, sizeof(float) * n, st));
    median_h_kernel<<<ceil_div(n, 256), 256, 0, st>>>(disp, W, H, tmp);
    note_launch();
    median_v_kernel<<<ceil_div(n, 256), 256, 0, st>>>(tmp, W, H, disp);
    note_launch();
    HBP_LAUNCH_CHECK();
}

} // namespace hbp
