// CPU oracle, post-processing (test infrastructure; see oracle_common.h).
// The reference's post-processing is itself CPU code (post_process.cu), so
// this restatement follows it operation for operation.
#include <algorithm>
#include <tuple>

#include "oracle_api.h"
#include "oracle_common.h"

namespace
{
// GetZ (post_process.cu:43-46)
inline float get_z(const float *v, int x, int y) { return v[0] * (float)x + v[1] * (float)y + v[2]; }
} // namespace

extern "C" {

// PostProcess::left_right_check (post_process.cu:47-110) with
// doConsistencyCheck (:4-41): a left pixel fails when the right disparity at
// int(x - d + 0.5f) differs by more than 1.5; the failure mask is dilated by a
// 3x3 box; every failed pixel takes the plane of the nearest non-dilated pixel
// to its left or right, whichever gives the smaller disparity at the pixel.
// planeL (HW x 3) is updated in place; failL receives the undilated mask
// (0/255) of the left view.
void orc_lr_check(const float *dispL, const float *dispR, float *planeL, int W, int H, uint8_t *failL)
{
    const int n = W * H;
    std::vector<uint8_t> fail(n, 0), fail2(n, 0);
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
        {
            float ds = dispL[y * W + x];
            if (ds != ds)
                continue;
            int rx = int((float)x - ds * 1.0f + 0.5f);
            if (rx >= 0 && rx < W)
            {
                float dsr = dispR[y * W + rx];
                if (std::fabs(dsr - ds) > 1.5)
                    fail[y * W + x] = 255;
            }
        }
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
        {
            uint8_t m = 0;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx)
                {
                    int yy = y + dy, xx = x + dx;
                    if (yy >= 0 && yy < H && xx >= 0 && xx < W)
                        m = std::max(m, fail[yy * W + xx]);
                }
            fail2[y * W + x] = m;
        }
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
        {
            if (!fail[y * W + x])
                continue;
            int xl = x, xr = x;
            while (xl >= 0 && fail2[y * W + xl] == 255)
                xl--;
            while (xr < W && fail2[y * W + xr] == 255)
                xr++;
            const float *pl = xl >= 0 ? planeL + 3 * (size_t)(y * W + xl) : nullptr;
            const float *pr = xr < W ? planeL + 3 * (size_t)(y * W + xr) : nullptr;
            const float *pick = nullptr;
            if (!pl && !pr)
                continue;
            else if (!pl)
                pick = pr;
            else if (!pr)
                pick = pl;
            else
                pick = get_z(pl, x, y) < get_z(pr, x, y) ? pl : pr;
            std::memcpy(planeL + 3 * (size_t)(y * W + x), pick, 12);
        }
    if (failL)
        std::memcpy(failL, fail.data(), n);
}

// PostProcess::plane_label_to_disp (post_process.cu:373-390): d = a*x + b*y + c.
void orc_plane_to_disp(const float *plane, int W, int H, float *disp)
{
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
            disp[y * W + x] = get_z(plane + 3 * (size_t)(y * W + x), x, y);
}

// PostProcess::median_filter (post_process.cu:112-185): for every failed left
// pixel, the colour-weighted median (weight exp(-sum|dBGR| / 10), window 41x41
// clipped to the image) of the window's planes ordered by their disparity at
// the pixel. stable != 0 orders equal disparities by window position (the
// engine's order); stable == 0 uses std::sort exactly as the reference does.
void orc_weighted_median(const uint8_t *bgr, const uint8_t *fail, float *plane, int W, int H,
                         int stable)
{
    std::vector<float> copy(plane, plane + 3 * (size_t)W * H);
    const int R = 20;
    const float omega = 10.0f;
    using Triplet = std::tuple<int, float, float>; // window sample, weight, z
#pragma omp parallel for schedule(dynamic, 16)
    for (int y = 0; y < H; ++y)
    {
        std::vector<Triplet> med;
        for (int x = 0; x < W; ++x)
        {
            if (!fail[y * W + x])
                continue;
            med.clear();
            double sumw = 0;
            int y0 = std::max(y - R, 0), y1 = std::min(y + R + 1, H);
            int x0 = std::max(x - R, 0), x1 = std::min(x + R + 1, W);
            const uint8_t *s = bgr + 3 * (size_t)(y * W + x);
            for (int yy = y0; yy < y1; ++yy)
                for (int xx = x0; xx < x1; ++xx)
                {
                    const uint8_t *t = bgr + 3 * (size_t)(yy * W + xx);
                    float a0 = (float)s[0] - (float)t[0], a1 = (float)s[1] - (float)t[1],
                          a2 = (float)s[2] - (float)t[2];
                    float absdiff = std::fabs(a0) + std::fabs(a1) + std::fabs(a2);
                    float w = std::exp(-absdiff / omega);
                    sumw += w;
                    int q = yy * W + xx;
                    med.emplace_back(q, w, get_z(copy.data() + 3 * (size_t)q, x, y));
                }
            auto cmp = [](const Triplet &a, const Triplet &b) { return std::get<2>(a) < std::get<2>(b); };
            if (stable)
                std::stable_sort(med.begin(), med.end(), cmp);
            else
                std::sort(med.begin(), med.end(), cmp);
            double center = sumw / 2.0;
            sumw = 0;
            for (size_t j = 0; j < med.size(); ++j)
            {
                sumw += std::get<1>(med[j]);
                if (sumw > center)
                {
                    std::memcpy(plane + 3 * (size_t)(y * W + x), copy.data() + 3 * (size_t)std::get<0>(med[j]), 12);
                    break;
                }
            }
        }
    }
}

// PostProcess::median_filter_gpu (post_process.cu:188-371), the reference's
// GPU variant of the weighted median, restated literally: per failed pixel the
// clipped 41x41 window in row-major order gives (window index, weight, z),
// the weight being compute_patch_weight's expf(-sum|dBGR| / 10) (wtab[k] for
// the integer colour distance k: the device's expf values, passed in), and
// z the plane's disparity at the pixel as the device evaluates
// a * x + b * y + c (z_mode 0: fma(a, x, b * y) + c; 1: unfused; 2:
// fma(a, x, fma(b, y, c))). The total weight is a float sum in window order;
// the samples are ordered by bubble_sort (:216-229: for each i, every later j
// with a smaller z is swapped into i), and the first sample whose float
// running weight exceeds half the total gives the plane. Position i is final
// once step i ends, so the scan runs alongside the sort and stops there.
void orc_weighted_median_gpu(const uint8_t *bgr, const uint8_t *fail, float *plane, int W, int H,
                             const float *wtab, int z_mode)
{
    std::vector<float> copy(plane, plane + 3 * (size_t)W * H);
    const int R = 20;
    struct S
    {
        float i, w, z;
    };
#pragma omp parallel for schedule(dynamic, 16)
    for (int y = 0; y < H; ++y)
    {
        std::vector<S> m;
        for (int x = 0; x < W; ++x)
        {
            if (!fail[y * W + x])
                continue;
            m.clear();
            const int y0 = std::max(y - R, 0), y1 = std::min(y + R, H - 1);
            const int x0 = std::max(x - R, 0), x1 = std::min(x + R, W - 1);
            const uint8_t *s = bgr + 3 * (size_t)(y * W + x);
            float sumw = 0.f;
            int k = 0;
            for (int yy = y0; yy <= y1; ++yy)
                for (int xx = x0; xx <= x1; ++xx, ++k)
                {
                    const uint8_t *t = bgr + 3 * (size_t)(yy * W + xx);
                    const int d = std::abs((int)s[0] - (int)t[0]) + std::abs((int)s[1] - (int)t[1]) +
                                  std::abs((int)s[2] - (int)t[2]);
                    const float w = wtab[d];
                    sumw += w;
                    const float *pl = copy.data() + 3 * (size_t)(yy * W + xx);
                    const float fx = (float)x, fy = (float)y;
                    float z;
                    if (z_mode == 0)
                        z = std::fma(pl[0], fx, pl[1] * fy) + pl[2];
                    else if (z_mode == 1)
                        z = (pl[0] * fx + pl[1] * fy) + pl[2];
                    else
                        z = std::fma(pl[0], fx, std::fma(pl[1], fy, pl[2]));
                    m.push_back({(float)k, w, z});
                }
            const int n = (int)m.size();
            const float center = sumw / 2;
            float run = 0.f;
            int pick = -1;
            for (int i = 0; i < n && pick < 0; ++i)
            {
                for (int j = i + 1; j < n; ++j)
                    if (m[j].z < m[i].z)
                        std::swap(m[i], m[j]);
                run += m[i].w;
                if (run > center)
                    pick = (int)m[i].i;
            }
            if (pick >= 0)
            {
                const int ww = x1 - x0 + 1;
                const int q = (y0 + pick / ww) * W + x0 + pick % ww;
                std::memcpy(plane + 3 * (size_t)(y * W + x), copy.data() + 3 * (size_t)q, 12);
            }
        }
    }
}

// medianFilter of the single-pair driver (main_stereo_hbp_isp.cu:120-192):
// a 7-tap horizontal median into a zero-initialised buffer over the interior
// (3-pixel border), then a 7-tap vertical median of that buffer back into D;
// pixels with D < 0 are copied instead. The vertical pass reads the buffer's
// untouched zero rows near the top and bottom borders, as the reference does.
void orc_driver_median(float *D, int W, int H)
{
    const int r = 3;
    std::vector<float> T((size_t)W * H, 0.0f);
    auto med7 = [](float *v) {
        // insertion sort as the reference (stable for equal values)
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
    };
    float v[7];
    for (int u = r; u < W - r; ++u)
        for (int y = r; y < H - r; ++y)
        {
            if (D[y * W + u] >= 0)
            {
                for (int k = 0; k < 7; ++k)
                    v[k] = D[y * W + u - r + k];
                T[y * W + u] = med7(v);
            }
            else
                T[y * W + u] = D[y * W + u];
        }
    for (int u = r; u < W - r; ++u)
        for (int y = r; y < H - r; ++y)
        {
            if (D[y * W + u] >= 0)
            {
                for (int k = 0; k < 7; ++k)
                    v[k] = T[(y - r + k) * W + u];
                D[y * W + u] = med7(v);
            }
        }
}

} // extern "C"
