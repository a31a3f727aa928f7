// CPU oracle, matching-cost and colour stages (test infrastructure; see
// oracle_common.h). Each function cites the reference code it restates.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "oracle_api.h"
#include "oracle_common.h"

using namespace orc;

extern "C" {

// img_BGR_to_grey + img_float1_to_uchar1 (imutil.cu:116-130, :154-168):
// g = B*0.114 + G*0.587 + R*0.299 in double, stored as float, truncated to u8
// (255 when g >= 255). The double sum is a multiple of 0.001 for integer
// inputs, so its rounding to float does not depend on the evaluation order.
void orc_grey_u8(const uint8_t *bgr, int n, uint8_t *out)
{
    for (int i = 0; i < n; ++i)
    {
        double g = bgr[3 * i] * 0.114 + bgr[3 * i + 1] * 0.587 + bgr[3 * i + 2] * 0.299;
        float f = (float)g;
        out[i] = f < 255.f ? (uint8_t)f : 255;
    }
}

// CenterSymmetricCensusKernelSM2 (stereo_cost.cu:45-146): 9x7 window, bit
// k*9+m = I(y-3+k, x-4+m) >= I(y+3-k, x+4-m) for k < 3, m < 9 and for k = 3,
// m < 4; pixels outside the image read 0.
void orc_census(const uint8_t *img, int W, int H, uint32_t *out)
{
    auto at = [&](int y, int x) -> int {
        return (y < 0 || x < 0 || y >= H || x >= W) ? 0 : img[y * W + x];
    };
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
        {
            uint32_t c = 0;
            for (int k = 0; k < 3; ++k)
                for (int m = 0; m < 9; ++m)
                    c |= (uint32_t)(at(y - 3 + k, x - 4 + m) >= at(y + 3 - k, x + 4 - m)) << (k * 9 + m);
            for (int m = 0; m < 4; ++m)
                c |= (uint32_t)(at(y, x - 4 + m) >= at(y, x + 4 - m)) << (27 + m);
            out[y * W + x] = c;
        }
}

// HammingDistanceCostKernel + cost_u1_to_f1_transpose + WTA_D_k
// (stereo_cost.cu:148-228, :248-280): V[d][p] = min(popc(cL[x] ^ cR[max(x-d,0)]), 25)
// for d < D, stored u8 disparity-major; wta = first argmin over d (strict <).
void orc_cost_volume(const uint32_t *cL, const uint32_t *cR, int W, int H, int D, uint8_t *vol,
                     float *wta)
{
    const size_t n = (size_t)W * H;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
        {
            size_t p = (size_t)y * W + x;
            float best = FLT_MAX;
            int arg = 0;
            for (int d = 0; d < D; ++d)
            {
                int xr = x - d < 0 ? 0 : x - d;
                int c = __builtin_popcount(cL[p] ^ cR[(size_t)y * W + xr]);
                uint8_t v = (uint8_t)(c < 25 ? c : 25);
                if (vol)
                    vol[(size_t)d * n + p] = v;
                if ((float)v < best)
                {
                    best = (float)v;
                    arg = d;
                }
            }
            if (wta)
                wta[p] = (float)arg;
        }
}

// StereoCost::compute_stereo_cost("MC-CNN") (stereo_cost.cu:436-444):
// read_volume_from_file (:396-418) copies the network's [D][H][W] volume,
// fill_out_of_view_k (:367-390, is_left) gives columns x <= d the value at
// x = d, truncate_data_k (:231-246) takes fminf(v, tau), and WTA_D_k
// (:249-266) keeps the first minimum. vol is [D][H*W] floats.
void orc_cost_f32(const float *src, int W, int H, int D, float tau, float *vol, float *wta)
{
    const size_t n = (size_t)W * H;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
        {
            float best = FLT_MAX;
            int arg = 0;
            for (int d = 0; d < D; ++d)
            {
                const float v = std::fmin(src[((size_t)d * H + y) * W + (x > d ? x : d)], tau);
                vol[(size_t)d * n + (size_t)y * W + x] = v;
                if (v < best)
                {
                    best = v;
                    arg = d;
                }
            }
            wta[(size_t)y * W + x] = (float)arg;
        }
}

// The same volume after StereoCost::cost_to_right (stereo_cost.cu:488-516),
// stated as the reference's three steps on the left volume: convert_vol_L2R_k
// (:471-486) moves each (d, y) row left by d in place, fill_out_of_view_k
// (:367-390, right side) copies column W-1-d over columns W-1-d .. W-1, and
// WTA_D_k keeps the first minimum.
static void float_volume_to_right(float *volR, int W, int H, int D, float *wta)
{
    const size_t n = (size_t)W * H;
    for (int d = 0; d < D; ++d)
        for (int y = 0; y < H; ++y)
        {
            float *row = volR + (size_t)d * n + (size_t)y * W;
            for (int x = 0; x + d < W; ++x)
                row[x] = row[x + d];
            const float c = row[W - 1 - d];
            for (int x = 0; x <= d; ++x)
                row[W - 1 - x] = c;
        }
    for (size_t p = 0; p < n; ++p)
    {
        float best = FLT_MAX;
        int arg = 0;
        for (int d = 0; d < D; ++d)
            if (volR[(size_t)d * n + p] < best)
            {
                best = volR[(size_t)d * n + p];
                arg = d;
            }
        wta[p] = (float)arg;
    }
}

void orc_cost_f32_right(const float *src, int W, int H, int D, float tau, float *volR, float *wta)
{
    std::vector<float> wl((size_t)W * H);
    orc_cost_f32(src, W, H, D, tau, volR, wl.data());
    float_volume_to_right(volR, W, H, D, wta);
}

// img_BGR_to_grey (imutil.cu:116-130): the double weighted sum stored as float.
void orc_grey_f32(const uint8_t *bgr, int n, float *out)
{
    for (int i = 0; i < n; ++i)
        out[i] = (float)(bgr[3 * i] * 0.114 + bgr[3 * i + 1] * 0.587 + bgr[3 * i + 2] * 0.299);
}

// compute_stereo_cost("AD") (stereo_cost.cu:421-429): ad_cost (:9-43) writes
// V[d][y][x] = fminf(fabsf(gL(x) - gR(x - d)), tau) for x >= D - 1 and 0 for
// every d where x < D - 1; WTA_D_k keeps the first minimum. right != 0 then
// applies cost_to_right (:488-516) as orc_cost_f32_right does.
void orc_cost_ad(const float *gL, const float *gR, int W, int H, int D, float tau, int right, float *vol,
                 float *wta)
{
    const size_t n = (size_t)W * H;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
        {
            const size_t i = (size_t)y * W + x;
            for (int d = 0; d < D; ++d)
                vol[(size_t)d * n + i] = x < D - 1 ? 0.0f : std::fmin(std::fabs(gL[i] - gR[i - d]), tau);
        }
    if (right)
    {
        float_volume_to_right(vol, W, H, D, wta);
        return;
    }
    for (size_t p = 0; p < n; ++p)
    {
        float best = FLT_MAX;
        int arg = 0;
        for (int d = 0; d < D; ++d)
            if (vol[(size_t)d * n + p] < best)
            {
                best = vol[(size_t)d * n + p];
                arg = d;
            }
        wta[p] = (float)arg;
    }
}

// StereoCost::cost_to_right (stereo_cost.cu:488-516): convert_vol_L2R_k shifts
// each (d, y) row left by d, fill_out_of_view_k repeats column W-1-d over the
// last d+1 columns; together VR[d][y][x] = VL[d][y][min(x+d, W-1)]. Then WTA.
void orc_cost_to_right(const uint8_t *volL, int W, int H, int D, uint8_t *volR, float *wta)
{
    const size_t n = (size_t)W * H;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
        {
            size_t p = (size_t)y * W + x;
            float best = FLT_MAX;
            int arg = 0;
            for (int d = 0; d < D; ++d)
            {
                int xs = std::min(x + d, W - 1);
                uint8_t v = volL[(size_t)d * n + (size_t)y * W + xs];
                if (volR)
                    volR[(size_t)d * n + p] = v;
                if ((float)v < best)
                {
                    best = (float)v;
                    arg = d;
                }
            }
            if (wta)
                wta[p] = (float)arg;
        }
}

// BGR_to_LAB (imutil.cu:4-40) after img_uchar3_to_float4 (imutil.cu:170-185):
// sRGB -> XYZ -> CIELAB in double, stored as float4 (L, a, b, 1). The
// reference's device code contracts the XYZ dot products and the affine steps
// into fused multiply-adds; the same fusion is written out here with std::fma.
// Device and host pow() may differ in the last double ulp; any resulting
// float difference is listed in the override table passed to
// orc_lab_set_overrides (produced by an exhaustive GPU sweep).
static std::vector<uint32_t> g_lab_override_keys;
static std::vector<float> g_lab_override_vals;

void orc_lab_set_overrides(const uint32_t *keys, const float *vals, int n)
{
    g_lab_override_keys.assign(keys, keys + n);
    g_lab_override_vals.assign(vals, vals + 3 * (size_t)n);
}

static inline void lab_of(float B, float G, float R, float W, float *o)
{
    double b = B / 255.0, g = G / 255.0, r = R / 255.0;
    r = (r > 0.04045) ? std::pow((r + 0.055) / 1.055, 2.4) : r / 12.92;
    g = (g > 0.04045) ? std::pow((g + 0.055) / 1.055, 2.4) : g / 12.92;
    b = (b > 0.04045) ? std::pow((b + 0.055) / 1.055, 2.4) : b / 12.92;
    double x = std::fma(b, 0.180423, std::fma(r, 0.412453, g * 0.357580)) / 0.950456;
    double y = std::fma(b, 0.072169, std::fma(r, 0.212671, g * 0.715160)) / 1.0;
    double z = std::fma(b, 0.950227, std::fma(r, 0.019334, g * 0.119193)) / 1.088754;
    const double eps = 216 / 24389.0, k = 841 / 108.0, kb = 16 / 116.0, third = 1 / 3.0;
    x = (x > eps) ? std::pow(x, third) : std::fma(k, x, kb);
    y = (y > eps) ? std::pow(y, third) : std::fma(k, y, kb);
    z = (z > eps) ? std::pow(z, third) : std::fma(k, z, kb);
    o[0] = (float)std::fma(116.0, y, -16.0);
    o[1] = (float)(500 * (x - y));
    o[2] = (float)(200 * (y - z));
    o[3] = W;
}

static inline void lab_one(uint8_t B, uint8_t G, uint8_t R, float *o) { lab_of(B, G, R, 1.0f, o); }

void orc_lab(const uint8_t *bgr, int n, float *lab4)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i)
    {
        lab_one(bgr[3 * i], bgr[3 * i + 1], bgr[3 * i + 2], lab4 + 4 * (size_t)i);
        if (!g_lab_override_keys.empty())
        {
            uint32_t key = (uint32_t)bgr[3 * i] | ((uint32_t)bgr[3 * i + 1] << 8) | ((uint32_t)bgr[3 * i + 2] << 16);
            auto it = std::lower_bound(g_lab_override_keys.begin(), g_lab_override_keys.end(), key);
            if (it != g_lab_override_keys.end() && *it == key)
            {
                size_t j = (size_t)(it - g_lab_override_keys.begin());
                lab4[4 * (size_t)i] = g_lab_override_vals[3 * j];
                lab4[4 * (size_t)i + 1] = g_lab_override_vals[3 * j + 1];
                lab4[4 * (size_t)i + 2] = g_lab_override_vals[3 * j + 2];
            }
        }
    }
}

// Pixel distance of compute_1nn_grid_k (segment.cu:14-22): |dLab|^2 + max(dL, 0),
// evaluated as the reference's device code does: fma(dz,dz, fma(dx,dx, dy*dy))
// followed by a rounded add of the hinge.
static inline float pix_dist(const float *s, const float *t)
{
    float dx = s[0] - t[0], dy = s[1] - t[1], dz = s[2] - t[2];
    float d = std::fma(dz, dz, std::fma(dx, dx, dy * dy));
    float h = dx > 0.f ? dx : 0.f;
    return d + h;
}

// compute_1nn_grid_k (segment.cu:57-195), 4-neighbour grid: neighbours in the
// order up, down, left, right; the first strict minimum wins. Also writes the
// level-0 directed edge list bd[4i+k] = (i, neighbour or i).
// SegHAC::img_CPU_to_GPU with sigma (segment.cu:795-809): the float4 image
// (B, G, R, 1), blurred when sigma > FLT_MIN by img_gauss_blur (imutil.cu:
// 397-497), then BGR -> LAB (which keeps the fourth channel). The blur: S =
// round(3 sigma); weights exp(-(r^2 + c^2) / (2 sigma^2)) in double, scaled by
// the reciprocal of their sum, stored as float; coordinates clamped to the
// image; per pixel the taps accumulate row by row (r outer, c inner) from 0 as
// sum = fma(pixel, weight, sum) per channel, the fused form of the
// reference's sum += pixel * weight. Pixels are those of a thread whose
// output position lies inside the image; the reference's edge blocks also let
// threads beyond a ragged right or bottom edge write the clamped last
// column/row, so only sizes that are multiples of 16 are deterministic there.
void orc_lab_sigma(const uint8_t *bgr, int W, int H, double sigma, float *lab4)
{
    const size_t n = (size_t)W * H;
    std::vector<float> img(4 * n);
    for (size_t i = 0; i < n; ++i)
    {
        img[4 * i] = bgr[3 * i];
        img[4 * i + 1] = bgr[3 * i + 1];
        img[4 * i + 2] = bgr[3 * i + 2];
        img[4 * i + 3] = 1.0f;
    }
    if (sigma > FLT_MIN)
    {
        const int S = (int)std::round(3 * sigma), F = 2 * S + 1;
        std::vector<double> w64((size_t)F * F);
        double sum = 0;
        for (int r = -S; r <= S; ++r)
            for (int c = -S; c <= S; ++c)
            {
                double v = std::exp(-(double)(r * r + c * c) / (2 * sigma * sigma));
                w64[(size_t)(r + S) * F + c + S] = v;
                sum += v;
            }
        sum = 1. / sum;
        std::vector<float> w((size_t)F * F);
        for (size_t k = 0; k < w.size(); ++k)
            w[k] = (float)(w64[k] * sum);
        std::vector<float> out(4 * n);
#pragma omp parallel for schedule(static)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x)
            {
                float acc[4] = {0, 0, 0, 0};
                for (int r = -S; r <= S; ++r)
                {
                    const int yy = std::min(std::max(y + r, 0), H - 1);
                    for (int c = -S; c <= S; ++c)
                    {
                        const int xx = std::min(std::max(x + c, 0), W - 1);
                        const float wt = w[(size_t)(r + S) * F + c + S];
                        const float *p = &img[4 * ((size_t)yy * W + xx)];
                        for (int ch = 0; ch < 4; ++ch)
                            acc[ch] = std::fma(p[ch], wt, acc[ch]);
                    }
                }
                for (int ch = 0; ch < 4; ++ch)
                    out[4 * ((size_t)y * W + x) + ch] = acc[ch];
            }
        img.swap(out);
    }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i)
        lab_of(img[4 * i], img[4 * i + 1], img[4 * i + 2], img[4 * i + 3], lab4 + 4 * i);
}

// compute_1nn_grid_k (segment.cu:57-195) with num_nb = 4 or 8: neighbours up,
// down, left, right, then up-left, up-right, down-right, down-left; first
// strict minimum. bd (2 ints per edge) and edist (the distance of each
// existing edge; missing neighbours give the self-edge (i, i)) are optional.
void orc_nn_grid_nb(const float *lab4, int W, int H, int num_nb, int *nn, float *dist_min, int *bd, float *edist)
{
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
        {
            int i = y * W + x;
            const float *s = lab4 + 4 * (size_t)i;
            float best = FLT_MAX;
            int arg = 0;
            const int nb[8] = {y > 0 ? i - W : -1,
                               y < H - 1 ? i + W : -1,
                               x > 0 ? i - 1 : -1,
                               x < W - 1 ? i + 1 : -1,
                               y > 0 && x > 0 ? i - W - 1 : -1,
                               y > 0 && x < W - 1 ? i - W + 1 : -1,
                               y < H - 1 && x < W - 1 ? i + W + 1 : -1,
                               y < H - 1 && x > 0 ? i + W - 1 : -1};
            for (int k = 0; k < num_nb; ++k)
            {
                const size_t e = (size_t)num_nb * i + k;
                if (bd)
                {
                    bd[2 * e] = i;
                    bd[2 * e + 1] = nb[k] < 0 ? i : nb[k];
                }
                if (edist)
                    edist[e] = 0.0f;
                if (nb[k] < 0)
                    continue;
                float d = pix_dist(s, lab4 + 4 * (size_t)nb[k]);
                if (edist)
                    edist[e] = d;
                if (d < best)
                {
                    best = d;
                    arg = nb[k];
                }
            }
            nn[i] = arg;
            dist_min[i] = best;
        }
}

void orc_nn_grid(const float *lab4, int W, int H, int *nn, float *dist_min, int *bd)
{
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
        {
            int i = y * W + x;
            const float *s = lab4 + 4 * (size_t)i;
            float best = FLT_MAX;
            int arg = 0;
            int nb[4] = {y > 0 ? i - W : -1, y < H - 1 ? i + W : -1, x > 0 ? i - 1 : -1,
                         x < W - 1 ? i + 1 : -1};
            for (int k = 0; k < 4; ++k)
            {
                if (bd)
                {
                    bd[2 * (4 * (size_t)i + k)] = i;
                    bd[2 * (4 * (size_t)i + k) + 1] = nb[k] < 0 ? i : nb[k];
                }
                if (nb[k] < 0)
                    continue;
                float d = pix_dist(s, lab4 + 4 * (size_t)nb[k]);
                if (d < best)
                {
                    best = d;
                    arg = nb[k];
                }
            }
            nn[i] = arg;
            dist_min[i] = best;
        }
}

} // extern "C"
