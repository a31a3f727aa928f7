// BGR -> CIELAB (L, a, b, 1) per pixel, in double precision as the
// reference does: img_uchar3_to_float4 + BGR_to_LAB (imutil.cu:4-40,
// :170-185, :330-340). The multiply-adds are fused exactly where the
// reference's device build fuses them (checked bit for bit against the
// reference build's output); pow is CUDA's double pow, as in the reference.
// This file is compiled with the default contraction setting so that pow's
// own arithmetic is the library's.
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
} // namespace

void launch_lab(const uint8_t *bgr, int n, float4 *lab, cudaStream_t st)
{
    lab_kernel<<<ceil_div(n, 256), 256, 0, st>>>(bgr, n, lab);
    note_launch();
    HBP_LAUNCH_CHECK();
}
} // namespace hbp
