// StereoCost with the reference's interface (stereo_cost.hpp:8-131): census
// matching cost of a rectified pair on the B200 engine (hbp_cost_census_d).
// Differences: "Census" is the one cost offered; g_img_cost_d() is the
// engine's uint8 volume in its tiled layout (hbp_volume_bytes), holding the
// same integer costs as the reference's float volume.
#pragma once

#include "common.hpp"

namespace hbp_isp
{
class StereoCost
{
  public:
    StereoCost(const Mat &img_left, const Mat &img_right, int labels, std::string vol_dir = "")
        : width(img_left.cols), height(img_left.rows), m_labels(labels), vol_dir(std::move(vol_dir))
    {
        detail::need_bgr(img_left, "StereoCost");
        detail::need_bgr(img_right, "StereoCost");
        if (img_right.cols != width || img_right.rows != height)
            throw std::invalid_argument("StereoCost: the two views differ in size");
        imgL = detail::upload(img_left);
        imgR = detail::upload(img_right);
    }

    // compute_stereo_cost (stereo_cost.cu:421-445)
    void compute_stereo_cost(const std::string &algo)
    {
        if (algo != "Census")
            throw std::invalid_argument("StereoCost: only the \"Census\" cost is offered");
        run(false);
    }

    // cost_to_right (stereo_cost.cu:488-516): the volume and WTA become the
    // right view's
    void cost_to_right() { run(true); }

    int g_labels() const { return m_labels; }
    int g_im_size() const { return width * height; }
    int g_width() const { return width; }
    int g_height() const { return height; }
    float g_tau() const { return 25.0f; }
    const uint8_t *g_img_cost_d() const { return vol ? vol->as<uint8_t>() : nullptr; }
    float *g_img_D_d() const { return wta ? wta->as<float>() : nullptr; }

    // shared with StereoData (which the reference deep-copies)
    detail::Buf vol, wta;

  private:
    void run(bool right)
    {
        const size_t n = (size_t)width * height;
        detail::Buf cL = std::make_shared<detail::DevBuf>(4 * n), cR = std::make_shared<detail::DevBuf>(4 * n);
        detail::Buf v = std::make_shared<detail::DevBuf>(hbp_volume_bytes(width, height, m_labels));
        detail::Buf w = std::make_shared<detail::DevBuf>(4 * n);
        detail::Buf vr, wr;
        if (right)
        {
            vr = std::make_shared<detail::DevBuf>(hbp_volume_bytes(width, height, m_labels));
            wr = std::make_shared<detail::DevBuf>(4 * n);
        }
        detail::check(hbp_cost_census_d(detail::shared_ctx()->h, imgL->as<uint8_t>(), imgR->as<uint8_t>(), width,
                                        height, m_labels, cL->as<uint32_t>(), cR->as<uint32_t>(),
                                        v->as<uint8_t>(), w->as<float>(), right ? vr->as<uint8_t>() : nullptr,
                                        right ? wr->as<float>() : nullptr, nullptr));
        vol = right ? vr : v;
        wta = right ? wr : w;
    }

    int width, height, m_labels;
    std::string vol_dir;
    detail::Buf imgL, imgR;
};
} // namespace hbp_isp

#ifndef HBP_ISP_NO_GLOBAL_NAMES
using hbp_isp::StereoCost;
#endif
