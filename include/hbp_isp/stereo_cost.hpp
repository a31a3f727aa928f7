// StereoCost with the reference's interface (stereo_cost.hpp:8-131): the
// matching cost of a rectified pair on the B200 engine.
//   "Census": hbp_cost_census_d; g_img_cost_d() is the engine's uint8 volume
//             in its tiled layout (hbp_volume_bytes), holding the same
//             integer costs as the reference's float volume.
//   "MC-CNN": the network's volume read from vol_dir (raw [D][H][W] floats,
//             as read_volume_from_file reads im0.acrt, stereo_cost.cu:396-418),
//             then hbp_cost_f32_d; g_img_cost_f32_d() is the tiled float
//             volume (hbp_volume_f32_bytes).
//   "AD":     hbp_cost_ad_d (truncation 30); the volume as for "MC-CNN".
// Any other name throws std::invalid_argument.
#pragma once

#include <fstream>

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
        if (algo == "Census")
        {
            f32 = false;
            m_tau = 25.0f;
            run(false);
        }
        else if (algo == "MC-CNN")
        {
            f32 = true;
            ad = false;
            m_tau = 0.5f;
            read_volume();
            run_f32(false);
        }
        else if (algo == "AD")
        {
            f32 = true;
            ad = true;
            m_tau = 30.0f;
            run_ad(false);
        }
        else
            throw std::invalid_argument("StereoCost: the \"Census\", \"MC-CNN\" and \"AD\" costs are offered");
    }

    // cost_to_right (stereo_cost.cu:488-516): the volume and WTA become the
    // right view's
    void cost_to_right()
    {
        if (ad)
            run_ad(true);
        else if (f32)
            run_f32(true);
        else
            run(true);
    }

    int g_labels() const { return m_labels; }
    int g_im_size() const { return width * height; }
    int g_width() const { return width; }
    int g_height() const { return height; }
    float g_tau() const { return m_tau; }
    bool g_is_f32() const { return f32; }
    const uint8_t *g_img_cost_d() const { return vol && !f32 ? vol->as<uint8_t>() : nullptr; }
    const float *g_img_cost_f32_d() const { return vol && f32 ? vol->as<float>() : nullptr; }
    float *g_img_D_d() const { return wta ? wta->as<float>() : nullptr; }

    // shared with StereoData (which the reference deep-copies)
    detail::Buf vol, wta;

  private:
    // read_volume_from_file (stereo_cost.cu:396-418): D x H x W floats, no header
    void read_volume()
    {
        const size_t bytes = sizeof(float) * (size_t)m_labels * width * height;
        std::ifstream f(vol_dir, std::ios::binary);
        if (!f)
            throw std::runtime_error("StereoCost: cost volume file " + vol_dir + " not found");
        std::vector<char> host(bytes);
        f.read(host.data(), (std::streamsize)bytes);
        if ((size_t)f.gcount() != bytes)
            throw std::runtime_error("StereoCost: cost volume file " + vol_dir + " is shorter than D x H x W floats");
        src = std::make_shared<detail::DevBuf>(bytes);
        detail::check(hbp_copy(src->p, host.data(), bytes));
    }

    void run_ad(bool right)
    {
        const size_t n = (size_t)width * height;
        detail::Buf gL = std::make_shared<detail::DevBuf>(4 * n), gR = std::make_shared<detail::DevBuf>(4 * n);
        detail::Buf v = std::make_shared<detail::DevBuf>(hbp_volume_f32_bytes(width, height, m_labels));
        detail::Buf w = std::make_shared<detail::DevBuf>(4 * n);
        detail::check(hbp_cost_ad_d(detail::shared_ctx()->h, imgL->as<uint8_t>(), imgR->as<uint8_t>(), width, height,
                                    m_labels, gL->as<float>(), gR->as<float>(), right ? nullptr : v->as<float>(),
                                    right ? nullptr : w->as<float>(), right ? v->as<float>() : nullptr,
                                    right ? w->as<float>() : nullptr, nullptr));
        vol = v;
        wta = w;
    }

    void run_f32(bool right)
    {
        const size_t n = (size_t)width * height;
        detail::Buf v = std::make_shared<detail::DevBuf>(hbp_volume_f32_bytes(width, height, m_labels));
        detail::Buf w = std::make_shared<detail::DevBuf>(4 * n);
        detail::check(hbp_cost_f32_d(detail::shared_ctx()->h, src->as<float>(), width, height, m_labels, m_tau,
                                     right ? nullptr : v->as<float>(), right ? nullptr : w->as<float>(),
                                     right ? v->as<float>() : nullptr, right ? w->as<float>() : nullptr, nullptr));
        vol = v;
        wta = w;
    }

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
    detail::Buf imgL, imgR, src;
    bool f32 = false, ad = false;
    float m_tau = 25.0f;
};
} // namespace hbp_isp

#ifndef HBP_ISP_NO_GLOBAL_NAMES
using hbp_isp::StereoCost;
#endif
