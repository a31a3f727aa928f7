// BGR -> CIELAB (L, a, b, 1) per pixel, in double precision as the
// reference does: img_uchar3_to_float4 + BGR_to_LAB (imutil.cu:4-40,
// :170-185, :330-340). The multiply-adds are fused exactly where the
// reference's device build fuses them (checked bit for bit against the
// reference build's output); pow is CUDA's double pow, as in the reference.
// This file is compiled with the default contraction setting so that pow's
// own arithmetic is the library's.
#include <cmath>

#include "engine.h"

namespace hbp
{
namespace
{
__global__ void lab_kernel(const uint8_t *__restrict__ bgr, int n, float4 *__restrict__ out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const uint8_t *p = bgr + 3 * (size_t)i;
    double b = (float)p[0] / 255.0, g = (float)p[1] / 255.0, r = (float)p[2] / 255.0;
    r = (r > 0.04045) ? pow((r + 0.055) / 1.055, 2.4) : r / 12.92;
    g = (g > 0.04045) ? pow((g + 0.055) / 1.055, 2.4) : g / 12.92;
    b = (b > 0.04045) ? pow((b + 0.055) / 1.055, 2.4) : b / 12.92;
    double x = fma(b, 0.180423, fma(r, 0.412453, g * 0.357580)) / 0.950456;
    double y = fma(b, 0.072169, fma(r, 0.212671, g * 0.715160)) / 1.0;
    double z = fma(b, 0.950227, fma(r, 0.019334, g * 0.119193)) / 1.088754;
    const double eps = 216 / 24389.0, k = 841 / 108.0, kb = 16 / 116.0, third = 1 / 3.0;
    x = (x > eps) ? pow(x, third) : fma(k, x, kb);
    y = (y > eps) ? pow(y, third) : fma(k, y, kb);
    z = (z > eps) ? pow(z, third) : fma(k, z, kb);
    float4 o;
    o.x = (float)fma(116.0, y, -16.0);
    o.y = (float)(500 * (x - y));
    o.z = (float)(200 * (y - z));
    o.w = 1.0f;
    out[i] = o;
}

// The same conversion on a float BGR image (the blurred image of SegHAC with
// sigma > 0); the fourth channel passes through (BGR_to_LAB keeps in.w).
__global__ void lab_f4_kernel(const float4 *__restrict__ in, int n, float4 *__restrict__ out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float4 v = in[i];
    double b = v.x / 255.0, g = v.y / 255.0, r = v.z / 255.0;
    r = (r > 0.04045) ? pow((r + 0.055) / 1.055, 2.4) : r / 12.92;
    g = (g > 0.04045) ? pow((g + 0.055) / 1.055, 2.4) : g / 12.92;
    b = (b > 0.04045) ? pow((b + 0.055) / 1.055, 2.4) : b / 12.92;
    double x = fma(b, 0.180423, fma(r, 0.412453, g * 0.357580)) / 0.950456;
    double y = fma(b, 0.072169, fma(r, 0.212671, g * 0.715160)) / 1.0;
    double z = fma(b, 0.950227, fma(r, 0.019334, g * 0.119193)) / 1.088754;
    const double eps = 216 / 24389.0, k = 841 / 108.0, kb = 16 / 116.0, third = 1 / 3.0;
    x = (x > eps) ? pow(x, third) : fma(k, x, kb);
    y = (y > eps) ? pow(y, third) : fma(k, y, kb);
    z = (z > eps) ? pow(z, third) : fma(k, z, kb);
    float4 o;
    o.x = (float)fma(116.0, y, -16.0);
    o.y = (float)(500 * (x - y));
    o.z = (float)(200 * (y - z));
    o.w = v.w;
    out[i] = o;
}

// Gaussian blur of the float4 image (B, G, R, 1) made from the BGR bytes:
// img_gauss_blur (imutil.cu:397-497). Per output pixel the (2S+1)^2 taps run
// row by row (r outer, c inner) on clamped coordinates, sum = fma(pixel,
// weight, sum) per channel from 0, the fused form of the reference's
// sum += pixel * weight.
struct BlurTaps
{
    int S;
    float w[(2 * BLUR_MAX_S + 1) * (2 * BLUR_MAX_S + 1)];
};

__global__ void blur_kernel(const uint8_t *__restrict__ bgr, int W, int H, BlurTaps taps, float4 *__restrict__ out)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H)
        return;
    const int S = taps.S, F = 2 * S + 1;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
    for (int r = -S; r <= S; ++r)
    {
        const int yy = min(max(y + r, 0), H - 1);
        for (int c = -S; c <= S; ++c)
        {
            const int xx = min(max(x + c, 0), W - 1);
            const float w = taps.w[(r + S) * F + c + S];
            const uint8_t *p = bgr + 3 * ((size_t)yy * W + xx);
            a0 = __fmaf_rn((float)p[0], w, a0);
            a1 = __fmaf_rn((float)p[1], w, a1);
            a2 = __fmaf_rn((float)p[2], w, a2);
            a3 = __fmaf_rn(1.0f, w, a3);
        }
    }
    out[(size_t)y * W + x] = make_float4(a0, a1, a2, a3);
}

// compute_patch_weight of median_filter_gpu (post_process.cu:199-213) for
// every colour distance k = 0..765: expf(-k / 10.0f), CUDA's expf as the
// reference's device code calls it (this file keeps the default contraction
// setting, so the library function is compiled as it is there).
__global__ void patch_weight_kernel(float *wtab)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < 766)
    {
        const float absdiff = (float)k;
        wtab[k] = expf(-absdiff / 10.0f);
    }
}
} // namespace

void launch_patch_weights(float *wtab766, cudaStream_t st)
{
    patch_weight_kernel<<<ceil_div(766, 128), 128, 0, st>>>(wtab766);
    note_launch();
    HBP_LAUNCH_CHECK();
}

int blur_radius(double sigma) { return (int)std::round(3 * sigma); }

void launch_lab_blur(const uint8_t *bgr, int W, int H, double sigma, float4 *tmp4, float4 *lab, cudaStream_t st)
{
    // compute_gauss_kernel (imutil.cu:443-473): weights in double on the
    // host, scaled by the reciprocal of their sum, stored as float
    BlurTaps taps{};
    const int S = blur_radius(sigma), F = 2 * S + 1;
    if (S > BLUR_MAX_S)
        throw StatusError{HBP_ERR_INVALID_ARG, "sigma too large: round(3 sigma) must be <= 7"};
    taps.S = S;
    double w64[(2 * BLUR_MAX_S + 1) * (2 * BLUR_MAX_S + 1)];
    double sum = 0;
    for (int r = -S; r <= S; ++r)
        for (int c = -S; c <= S; ++c)
        {
            double v = std::exp(-(double)(r * r + c * c) / (2 * sigma * sigma));
            w64[(r + S) * F + c + S] = v;
            sum += v;
        }
    sum = 1. / sum;
    for (int k = 0; k < F * F; ++k)
        taps.w[k] = (float)(w64[k] * sum);
    dim3 b(32, 8), g(ceil_div(W, 32), ceil_div(H, 8));
    blur_kernel<<<g, b, 0, st>>>(bgr, W, H, taps, tmp4);
    note_launch();
    HBP_LAUNCH_CHECK();
    const int n = W * H;
    lab_f4_kernel<<<ceil_div(n, 256), 256, 0, st>>>(tmp4, n, lab);
    note_launch();
    HBP_LAUNCH_CHECK();
}

void launch_lab(const uint8_t *bgr, int n, float4 *lab, cudaStream_t st)
{
    lab_kernel<<<ceil_div(n, 256), 256, 0, st>>>(bgr, n, lab);
    note_launch();
    HBP_LAUNCH_CHECK();
}
} // namespace hbp
