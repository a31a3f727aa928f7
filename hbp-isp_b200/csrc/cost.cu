// Matching cost: grey + 9x7 centre-symmetric census for both views, Hamming
// cost volume (uint8, disparity-major, clamped at tau = 25) and WTA.
//
// Reference: StereoCost::compute_stereo_cost("Census") (stereo_cost.cu:421-445)
// = img_BGR_to_grey + img_float1_to_uchar1 (imutil.cu:116-168),
// CenterSymmetricCensusKernelSM2 (stereo_cost.cu:45-146),
// HammingDistanceCostKernel (:148-207), cost_u1_to_f1_transpose (:209-228),
// WTA_D_k (:248-280); right view: cost_to_right (:471-516).
//
// Layout: pixel-major vol[y][x][d] with Dp = round_up(D, 16) bytes per pixel
// (entries d >= D are 0), so the data-cost kernel finds V[d] and V[d+1] of all
// of a pixel's candidate planes in one 32-byte sector. Values are
// min(popcount, 25) (exact in 8 bits; the reference's float volume holds the
// same integers).
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

constexpr int HM_THREADS = 128; // one pixel per thread, 128 pixels per block

// One block = 128 consecutive pixels of a row; thread = pixel. Shared memory
// holds the left census of the segment plus D columns to the right (right
// view) and the right census of the segment plus D columns to the left
// (clamped at the image border, which reproduces the reference's use of
// cR[row][0] for x-d < 0). Each thread writes its Dp cost bytes contiguously
// in 16-byte words (pixel-major, like the reference's u8 volume
// [px][D_align]).
__global__ void __launch_bounds__(HM_THREADS)
    hamming_wta_kernel(const uint32_t *__restrict__ cL, const uint32_t *__restrict__ cR, int W,
                       int H, int D, int Dp, uint8_t *__restrict__ vol, float *__restrict__ wta,
                       uint8_t *__restrict__ volR, float *__restrict__ wtaR)
{
    extern __shared__ uint32_t sm[];
    const int y = blockIdx.y;
    const int xs = blockIdx.x * HM_THREADS;
    const int span = HM_THREADS + D;
    uint32_t *sLc = sm;        // cL[xs + i], i in [0, span)  (clamped to W-1)
    uint32_t *sRc = sm + span; // cR[xs - D + i], i in [0, span) (clamped to 0 / W-1)
    const uint32_t *rowL = cL + (size_t)y * W, *rowR = cR + (size_t)y * W;
    for (int i = threadIdx.x; i < span; i += HM_THREADS)
    {
        int gl = min(xs + i, W - 1);
        int gr = max(min(xs - D + i, W - 1), 0);
        sLc[i] = rowL[gl];
        sRc[i] = rowR[gr];
    }
    __syncthreads();
    const int lx = threadIdx.x, x = xs + lx;
    if (x >= W)
        return;
    const size_t px = (size_t)y * W + x;
    const uint32_t cl = sLc[lx];
    uint4 *out = reinterpret_cast<uint4 *>(vol + px * Dp);
    int best = 1 << 30, arg = 0;
    for (int d0 = 0; d0 < Dp; d0 += 16)
    {
        uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
        for (int j = 0; j < 16; ++j)
        {
            int d = d0 + j;
            int c = 0;
            if (d < D)
            {
                // cR[max(x - d, 0)]: local index (lx - d) + D in sRc
                c = __popc(cl ^ sRc[lx - d + D]);
                c = c < 25 ? c : 25;
                if (c < best)
                {
                    best = c;
                    arg = d;
                }
            }
            w[j >> 2] |= (uint32_t)c << (8 * (j & 3));
        }
        out[d0 >> 4] = make_uint4(w[0], w[1], w[2], w[3]);
    }
    wta[px] = (float)arg;
    if (!volR)
        return;
    // Right view: VR[y][x][d] = V[y][min(x + d, W - 1)][d] (convert_vol_L2R_k
    // followed by fill_out_of_view_k).
    uint4 *outR = reinterpret_cast<uint4 *>(volR + px * Dp);
    best = 1 << 30;
    arg = 0;
    for (int d0 = 0; d0 < Dp; d0 += 16)
    {
        uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
        for (int j = 0; j < 16; ++j)
        {
            int d = d0 + j;
            int c = 0;
            if (d < D)
            {
                int xl = min(x + d, W - 1); // source column in the left view
                int xr = max(xl - d, 0);    // its match in the right view
                c = __popc(sLc[xl - xs] ^ sRc[xr - xs + D]);
                c = c < 25 ? c : 25;
                if (c < best)
                {
                    best = c;
                    arg = d;
                }
            }
            w[j >> 2] |= (uint32_t)c << (8 * (j & 3));
        }
        outR[d0 >> 4] = make_uint4(w[0], w[1], w[2], w[3]);
    }
    wtaR[px] = (float)arg;
}

} // namespace

int volume_pitch(int D) { return (D + 15) / 16 * 16; }

void launch_cost(const uint8_t *bgrL, const uint8_t *bgrR, int W, int H, int D, uint32_t *cL,
                 uint32_t *cR, uint8_t *vol, float *wta, uint8_t *volR, float *wtaR,
                 cudaStream_t st)
{
    dim3 cb(CT_W, CT_H), cg(ceil_div(W, CT_W), ceil_div(H, CT_H));
    census_pair_kernel<<<cg, cb, 0, st>>>(bgrL, bgrR, W, H, cL, cR);
    note_launch();
    HBP_LAUNCH_CHECK();
    const int Dp = volume_pitch(D);
    size_t smem = sizeof(uint32_t) * 2 * (HM_THREADS + D);
    dim3 hg(ceil_div(W, HM_THREADS), H);
    hamming_wta_kernel<<<hg, HM_THREADS, smem, st>>>(cL, cR, W, H, D, Dp, vol, wta, volR, wtaR);
    note_launch();
    HBP_LAUNCH_CHECK();
}

} // namespace hbp
