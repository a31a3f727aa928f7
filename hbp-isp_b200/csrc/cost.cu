// Matching cost: grey + 9x7 centre-symmetric census for both views, Hamming
// cost volume (uint8, disparity-major, clamped at tau = 25) and WTA.
//
// Reference: StereoCost::compute_stereo_cost("Census") (stereo_cost.cu:421-445)
// = img_BGR_to_grey + img_float1_to_uchar1 (imutil.cu:116-168),
// CenterSymmetricCensusKernelSM2 (stereo_cost.cu:45-146),
// HammingDistanceCostKernel (:148-207), cost_u1_to_f1_transpose (:209-228),
// WTA_D_k (:248-280); right view: cost_to_right (:471-516).
//
// Layout: 8x4-pixel tiles, disparity-major inside a tile (vol_offset in
// engine.h): one 32-byte sector holds a whole tile at one disparity, so the
// data-cost kernel, whose warps walk compact superpixels, touches few sectors
// per load. Values are min(popcount, 25) (exact in 8 bits; the reference's
// float volume holds the same integers).
#include <cfloat>

#include "engine.h"

namespace hbp
{

namespace
{
constexpr int CT_W = 32, CT_H = 8; // census tile
constexpr int HALO_X = 4, HALO_Y = 3;
constexpr int SW = CT_W + 2 * HALO_X, SH = CT_H + 2 * HALO_Y;

// grey = truncate(float(B*0.114 + G*0.587 + R*0.299)), capped at 255. The
// double sum equals k/1000 for the integer k = 114B + 587G + 299R and its
// nearest float lies within 2e-5 of it, while k/1000 is either an integer or
// at least 0.001 away from one; the truncation is therefore exactly k / 1000.
__device__ __forceinline__ uint8_t grey_of(const uint8_t *p)
{
    int k = 114 * p[0] + 587 * p[1] + 299 * p[2];
    int g = k / 1000;
    return (uint8_t)(g < 255 ? g : 255);
}

__global__ void __launch_bounds__(CT_W *CT_H)
    census_pair_kernel(const uint8_t *__restrict__ bgrL, const uint8_t *__restrict__ bgrR, int W,
                       int H, uint32_t *__restrict__ cL, uint32_t *__restrict__ cR)
{
    __shared__ uint8_t sL[SH][SW], sR[SH][SW];
    const int x0 = blockIdx.x * CT_W - HALO_X, y0 = blockIdx.y * CT_H - HALO_Y;
    const int tid = threadIdx.y * CT_W + threadIdx.x;
    for (int i = tid; i < SW * SH; i += CT_W * CT_H)
    {
        int sy = i / SW, sx = i % SW;
        int gx = x0 + sx, gy = y0 + sy;
        uint8_t l = 0, r = 0;
        if (gx >= 0 && gy >= 0 && gx < W && gy < H)
        {
            size_t o = 3 * ((size_t)gy * W + gx);
            l = grey_of(bgrL + o);
            r = grey_of(bgrR + o);
        }
        sL[sy][sx] = l;
        sR[sy][sx] = r;
    }
    __syncthreads();
    const int x = blockIdx.x * CT_W + threadIdx.x, y = blockIdx.y * CT_H + threadIdx.y;
    if (x >= W || y >= H)
        return;
    const int tx = threadIdx.x, ty = threadIdx.y;
    uint32_t a = 0, b = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int m = 0; m < 9; ++m)
        {
            a |= (uint32_t)(sL[ty + k][tx + m] >= sL[ty + 6 - k][tx + 8 - m]) << (k * 9 + m);
            b |= (uint32_t)(sR[ty + k][tx + m] >= sR[ty + 6 - k][tx + 8 - m]) << (k * 9 + m);
        }
#pragma unroll
    for (int m = 0; m < 4; ++m)
    {
        a |= (uint32_t)(sL[ty + 3][tx + m] >= sL[ty + 3][tx + 8 - m]) << (27 + m);
        b |= (uint32_t)(sR[ty + 3][tx + m] >= sR[ty + 3][tx + 8 - m]) << (27 + m);
    }
    cL[(size_t)y * W + x] = a;
    cR[(size_t)y * W + x] = b;
}

constexpr int HM_TILES = 8;               // 8x4-pixel tiles per block (one warp each)
constexpr int HM_THREADS = 32 * HM_TILES;  // 256
constexpr int HM_COLS = VT_W * HM_TILES;   // 64 columns x VT_H rows per block

// Shared-memory row stride of the census staging: >= HM_COLS + D and = 8
// (mod 32), so the four rows of a warp's tile fall in distinct banks.
__host__ __device__ inline int hm_stride(int D) { return (HM_COLS + D + 31) / 32 * 32 + 8; }

// One block = a strip of 64 columns x 4 rows (8 tiles); warp w = tile w, lane
// = (y & 3) * 8 + (x & 7). Shared memory holds, per row, the left census of
// the strip plus D columns to the right (right view) and the right census of
// the strip plus D columns to the left, clamped at the image border (which
// reproduces the reference's use of cR[row][0] for x-d < 0). For every d the
// warp stores its tile's 32 cost bytes as one sector; pixels outside the image
// get 0.
__global__ void __launch_bounds__(HM_THREADS)
    hamming_wta_kernel(const uint32_t *__restrict__ cL, const uint32_t *__restrict__ cR, int W,
                       int H, int D, int TX, uint8_t *__restrict__ vol, float *__restrict__ wta,
                       uint8_t *__restrict__ volR, float *__restrict__ wtaR)
{
    extern __shared__ uint32_t sm[];
    const int xs = blockIdx.x * HM_COLS, ys = blockIdx.y * VT_H;
    const int S = hm_stride(D), span = HM_COLS + D;
    uint32_t *sLc = sm;              // [VT_H][S]: cL[y][xs + i]
    uint32_t *sRc = sm + VT_H * S;   // [VT_H][S]: cR[y][xs - D + i]
    for (int r = 0; r < VT_H; ++r)
    {
        const int yy = min(ys + r, H - 1);
        const uint32_t *rowL = cL + (size_t)yy * W, *rowR = cR + (size_t)yy * W;
        for (int i = threadIdx.x; i < span; i += HM_THREADS)
        {
            sLc[r * S + i] = rowL[min(xs + i, W - 1)];
            sRc[r * S + i] = rowR[max(min(xs - D + i, W - 1), 0)];
        }
    }
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tx = (xs >> 3) + w;
    if (tx >= TX)
        return;
    const int ly = lane >> 3, lc = w * VT_W + (lane & 7);
    const int x = xs + lc, y = ys + ly;
    const bool in = x < W && y < H;
    const uint32_t *rL = sLc + ly * S, *rR = sRc + ly * S;
    const size_t tile = (size_t)blockIdx.y * TX + tx;
    uint8_t *out = vol + tile * D * VT_BYTES + lane;
    const uint32_t cl = rL[lc];
    int best = 1 << 30, arg = 0;
    for (int d = 0; d < D; ++d)
    {
        int c = 0;
        if (in)
        {
            // cR[max(x - d, 0)]: local index (lc - d) + D in rR
            c = __popc(cl ^ rR[lc - d + D]);
            c = c < 25 ? c : 25;
            if (c < best)
            {
                best = c;
                arg = d;
            }
        }
        out[(size_t)d * VT_BYTES] = (uint8_t)c;
    }
    if (in)
        wta[(size_t)y * W + x] = (float)arg;
    if (!volR)
        return;
    // Right view: VR(x, y, d) = V(min(x + d, W - 1), y, d) (convert_vol_L2R_k
    // followed by fill_out_of_view_k).
    uint8_t *outR = volR + tile * D * VT_BYTES + lane;
    best = 1 << 30;
    arg = 0;
    for (int d = 0; d < D; ++d)
    {
        int c = 0;
        if (in)
        {
            int xl = min(x + d, W - 1); // source column in the left view
            int xr = max(xl - d, 0);    // its match in the right view
            c = __popc(rL[xl - xs] ^ rR[xr - xs + D]);
            c = c < 25 ? c : 25;
            if (c < best)
            {
                best = c;
                arg = d;
            }
        }
        outR[(size_t)d * VT_BYTES] = (uint8_t)c;
    }
    if (in)
        wtaR[(size_t)y * W + x] = (float)arg;
}

// The MC-CNN volume ingest (stereo_cost.cu:396-418 and WTA_D_k, :249-266):
// src is the network's [D][H][W] float volume. Pixels left of the first
// valid column (x <= d) take the value at x = d (fill_out_of_view_k with
// is_left), every value is truncated at tau, and WTA keeps the first minimum.
// RIGHT: the same volume after cost_to_right (:488-516): convert_vol_L2R_k
// shifts each (d, y) row left by d and fill_out_of_view_k repeats column
// W-1-d to the right, so VR[d][y][x] = VL[d][y][min(x + d, W - 1)], which is
// min(src[d][y][min(x + d, W - 1)], tau) because min(x + d, W - 1) >= d.
// Same block and tile geometry as the Hamming kernel: warp w writes tile w of
// a 64x4 strip, 32 consecutive floats per disparity; each lane reads its row
// segment of eight columns (32-byte sectors).
template <bool RIGHT>
__global__ void __launch_bounds__(HM_THREADS)
    ingest_f32_kernel(const float *__restrict__ src, int W, int H, int D, float tau, int TX,
                      float *__restrict__ vol, float *__restrict__ wta)
{
    const int xs = blockIdx.x * HM_COLS, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tx = (xs >> 3) + w;
    if (tx >= TX)
        return;
    const int x = xs + w * VT_W + (lane & 7), y = blockIdx.y * VT_H + (lane >> 3);
    const bool in = x < W && y < H;
    float *out = vol + ((size_t)blockIdx.y * TX + tx) * D * VT_BYTES + lane;
    const float *row = src + (size_t)(in ? y : 0) * W;
    const size_t plane = (size_t)H * W;
    float best = FLT_MAX;
    int arg = 0;
#pragma unroll 4
    for (int d = 0; d < D; ++d)
    {
        float v = 0.0f;
        if (in)
        {
            v = fminf(__ldg(row + (size_t)d * plane + (RIGHT ? min(x + d, W - 1) : max(x, d))), tau);
            if (v < best)
            {
                best = v;
                arg = d;
            }
        }
        out[(size_t)d * VT_BYTES] = v;
    }
    if (in)
        wta[(size_t)y * W + x] = (float)arg;
}

// img_BGR_to_grey (imutil.cu:116-130) for both views: the float nearest to
// B*0.114 + G*0.587 + R*0.299. That double sum lies within 1e-13 of k/1000
// (k = 114B + 587G + 299R), and k/1000 is at least 7e-9 away from the
// midpoint of two floats below 256 (such a midpoint is an odd multiple of
// 2^-17 or finer, which k/1000 never is), so rounding the double sum and
// rounding k/1000 itself give the same float: the correctly rounded quotient.
__global__ void grey_f32_kernel(const uint8_t *__restrict__ bgrL, const uint8_t *__restrict__ bgrR, int n,
                                float *__restrict__ gL, float *__restrict__ gR)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const uint8_t *l = bgrL + 3 * (size_t)i, *r = bgrR + 3 * (size_t)i;
    gL[i] = __fdiv_rn((float)(114 * l[0] + 587 * l[1] + 299 * l[2]), 1000.0f);
    gR[i] = __fdiv_rn((float)(114 * r[0] + 587 * r[1] + 299 * r[2]), 1000.0f);
}

// ad_cost (stereo_cost.cu:9-43) and WTA_D_k: V[d][y][x] = min(|gL(x) - gR(x - d)|,
// tau) for x >= D - 1, and 0 for every d where x < D - 1 (the reference's
// border). RIGHT: the volume after cost_to_right, VR[d][y][x] =
// V[d][y][min(x + d, W - 1)]. Tiled float layout, geometry as the ingest.
template <bool RIGHT>
__global__ void __launch_bounds__(HM_THREADS)
    ad_volume_kernel(const float *__restrict__ gL, const float *__restrict__ gR, int W, int H, int D, float tau,
                     int TX, float *__restrict__ vol, float *__restrict__ wta)
{
    const int xs = blockIdx.x * HM_COLS, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tx = (xs >> 3) + w;
    if (tx >= TX)
        return;
    const int x = xs + w * VT_W + (lane & 7), y = blockIdx.y * VT_H + (lane >> 3);
    const bool in = x < W && y < H;
    float *out = vol + ((size_t)blockIdx.y * TX + tx) * D * VT_BYTES + lane;
    const float *rowL = gL + (size_t)(in ? y : 0) * W, *rowR = gR + (size_t)(in ? y : 0) * W;
    const float ref = in && !RIGHT ? __ldg(rowL + x) : 0.0f;
    float best = FLT_MAX;
    int arg = 0;
#pragma unroll 4
    for (int d = 0; d < D; ++d)
    {
        float v = 0.0f;
        if (in)
        {
            const int xl = RIGHT ? min(x + d, W - 1) : x; // the left-view column read
            if (xl >= D - 1)
                v = fminf(fabsf((RIGHT ? __ldg(rowL + xl) : ref) - __ldg(rowR + xl - d)), tau);
            if (v < best)
            {
                best = v;
                arg = d;
            }
        }
        out[(size_t)d * VT_BYTES] = v;
    }
    if (in)
        wta[(size_t)y * W + x] = (float)arg;
}
} // namespace

void launch_cost_ad(const uint8_t *bgrL, const uint8_t *bgrR, int W, int H, int D, float tau, float *greyL,
                    float *greyR, float *vol, float *wta, float *volR, float *wtaR, cudaStream_t st)
{
    const int n = W * H;
    grey_f32_kernel<<<ceil_div(n, 256), 256, 0, st>>>(bgrL, bgrR, n, greyL, greyR);
    note_launch();
    HBP_LAUNCH_CHECK();
    const int TX = ceil_div(W, VT_W);
    dim3 g(ceil_div(W, HM_COLS), ceil_div(H, VT_H));
    if (vol)
    {
        ad_volume_kernel<false><<<g, HM_THREADS, 0, st>>>(greyL, greyR, W, H, D, tau, TX, vol, wta);
        note_launch();
        HBP_LAUNCH_CHECK();
    }
    if (volR)
    {
        ad_volume_kernel<true><<<g, HM_THREADS, 0, st>>>(greyL, greyR, W, H, D, tau, TX, volR, wtaR);
        note_launch();
        HBP_LAUNCH_CHECK();
    }
}

void launch_ingest_f32(const float *src, int W, int H, int D, float tau, float *vol, float *wta, float *volR,
                       float *wtaR, cudaStream_t st)
{
    const int TX = ceil_div(W, VT_W);
    dim3 g(ceil_div(W, HM_COLS), ceil_div(H, VT_H));
    if (vol)
    {
        ingest_f32_kernel<false><<<g, HM_THREADS, 0, st>>>(src, W, H, D, tau, TX, vol, wta);
        note_launch();
        HBP_LAUNCH_CHECK();
    }
    if (volR)
    {
        ingest_f32_kernel<true><<<g, HM_THREADS, 0, st>>>(src, W, H, D, tau, TX, volR, wtaR);
        note_launch();
        HBP_LAUNCH_CHECK();
    }
}

void launch_cost(const uint8_t *bgrL, const uint8_t *bgrR, int W, int H, int D, uint32_t *cL,
                 uint32_t *cR, uint8_t *vol, float *wta, uint8_t *volR, float *wtaR,
                 cudaStream_t st)
{
    dim3 cb(CT_W, CT_H), cg(ceil_div(W, CT_W), ceil_div(H, CT_H));
    census_pair_kernel<<<cg, cb, 0, st>>>(bgrL, bgrR, W, H, cL, cR);
    note_launch();
    HBP_LAUNCH_CHECK();
    const int TX = ceil_div(W, VT_W);
    size_t smem = sizeof(uint32_t) * 2 * VT_H * hm_stride(D);
    dim3 hg(ceil_div(W, HM_COLS), ceil_div(H, VT_H));
    hamming_wta_kernel<<<hg, HM_THREADS, smem, st>>>(cL, cR, W, H, D, TX, vol, wta, volR, wtaR);
    note_launch();
    HBP_LAUNCH_CHECK();
}

} // namespace hbp
