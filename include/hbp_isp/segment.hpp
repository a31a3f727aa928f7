// SegHAC with the reference's interface (segment.hpp:8-27, :248): the image
// segmentation pyramid on the B200 engine (hbp_segment_target_d). Offered:
// every linkage (CentoridLink is the reference's spelling), 4 or 8
// neighbours, sigma with round(3 sigma) <= 7, every output format, the full
// hierarchy (target_clus 1) or target_clus superpixels; the cycle-root
// display (show_cycle) is rejected. Each SegHAC owns the engine context that
// holds its pyramid; ISPData shares it.
#pragma once

#include <cmath>

#include "common.hpp"

namespace hbp_isp
{
enum Linkage
{
    MinLink,
    MaxLink,
    CentoridLink,
    WardLink
};

enum SegFormat
{
    LabelUchar3Format,
    LabelIntFormat,
    BoundaryFormat,
    LabelDeviceIntFormat,
    LabelISPFormat,
    EmptyFormat
};

class SegHAC
{
  public:
    SegHAC(const Mat &src, Linkage link, int num_nb, double sigma, SegFormat seg_format, int target_clus,
           bool show_cycle)
        : width(src.cols), height(src.rows), m_link(link), m_num_nb(num_nb), m_sigma(sigma)
    {
        detail::need_bgr(src, "SegHAC");
        if (seg_format < LabelUchar3Format || seg_format > EmptyFormat)
            throw std::invalid_argument("SegHAC: unknown output format");
        if (target_clus < 1 || (long)target_clus >= (long)width * height)
            throw std::invalid_argument("SegHAC: target_clus must lie in [1, pixels)");
        if (show_cycle)
            throw std::invalid_argument("SegHAC: the cycle-root display is not offered");
        if (link < MinLink || link > WardLink || (num_nb != 4 && num_nb != 8) || !(sigma >= 0.0) ||
            (int)std::round(3 * sigma) > 7)
            throw std::invalid_argument("SegHAC: linkage Min/Max/Centroid/Ward, 4 or 8 neighbours, "
                                        "round(3 sigma) <= 7");
        m_format = seg_format;
        m_target = target_clus;
        img = detail::upload(src);
        ctx = std::make_shared<detail::Ctx>();
    }

    // run_ms (segment.cu:1279-1321) with save_output's pictures (:1096-1111):
    // LabelISPFormat and EmptyFormat leave segs untouched; the other formats
    // append one picture per level with target_clus 1, else one of the
    // target_clus superpixels. LabelUchar3Format and BoundaryFormat give
    // CV_8UC3 pictures, LabelIntFormat CV_32SC1 (labels from 1), and
    // LabelDeviceIntFormat, which the reference draws nothing for, empty
    // Mats. Each run builds the pyramid from the current image anew.
    void run_ms(std::vector<Mat> *segs = nullptr)
    {
        detail::check(hbp_segment_target_d(ctx->h, img->as<uint8_t>(), width, height, (int)m_link, m_num_nb,
                                           m_sigma, m_target, &levels, nullptr));
        if (m_format == LabelISPFormat || m_format == EmptyFormat)
            return;
        if (!segs)
            throw std::invalid_argument("SegHAC::run_ms: this output format needs a picture list");
        for (int l = m_target == 1 ? 0 : levels - 1; l < levels; ++l)
        {
            if (m_format == LabelDeviceIntFormat)
            {
                segs->emplace_back();
                continue;
            }
            Mat pic(height, width, m_format == LabelIntFormat ? MAT_32SC1 : MAT_8UC3);
            detail::DevBuf out(pic.bytes());
            detail::check(hbp_segment_draw_d(ctx->h, l, (int)m_format, img->as<uint8_t>(), out.p, nullptr));
            detail::check(hbp_copy(pic.data, out.p, pic.bytes()));
            segs->push_back(pic);
        }
    }

    // set_frame (segment.hpp:87-91): the next image of a video stream, same size
    void set_frame(const Mat &frame)
    {
        detail::need_bgr(frame, "SegHAC::set_frame");
        if (frame.cols != width || frame.rows != height)
            throw std::invalid_argument("SegHAC::set_frame: the frame size differs");
        img = detail::upload(frame);
    }
    // set_seq_img (segment.hpp:95-107): the next image of a sequence, same size
    // or transposed
    void set_seq_img(const Mat &frame)
    {
        detail::need_bgr(frame, "SegHAC::set_seq_img");
        if (frame.cols != width)
        {
            if (frame.cols != height || frame.rows != width)
                throw std::invalid_argument("SegHAC::set_seq_img: the image is neither the same size nor transposed");
            width = frame.cols;
            height = frame.rows;
        }
        img = detail::upload(frame);
    }

    int g_width() const { return width; }
    int g_height() const { return height; }
    int g_levels() const { return levels; }
    int g_mean_channels() const { return 6; }
    // the level sizes and the ISP arrays in place on the device (segment.hpp:
    // 118-150); the pointers stay valid until the next run_ms
    std::vector<int> g_num_clus_isp() const { return level_column(0); }
    std::vector<int> g_num_bd_isp() const { return level_column(1); }
    const int *g_isp_clus_d() const { return device_arrays().clus; }
    const float *g_isp_mean_d() const { return device_arrays().mean; }
    const int *g_isp_bd_d() const { return device_arrays().bd; }
    const int *g_isp_bdl_d() const { return device_arrays().bdl; }

    detail::CtxPtr ctx; // holds the pyramid after run_ms

  private:
    std::vector<int> level_column(int k) const
    {
        std::vector<int> sizes(2 * 64), out;
        detail::check(hbp_pyramid_levels(ctx->h, sizes.data(), 64));
        for (int l = 0; l < 64 && sizes[2 * l] > 0; ++l)
            out.push_back(sizes[2 * l + k]);
        return out;
    }
    struct DeviceArrays
    {
        const int *clus = nullptr;
        const float *mean = nullptr;
        const int *bd = nullptr, *bdl = nullptr;
    };
    DeviceArrays device_arrays() const
    {
        DeviceArrays a;
        detail::check(hbp_pyramid_device(ctx->h, &a.clus, &a.mean, &a.bd, &a.bdl));
        return a;
    }

    int width, height;
    Linkage m_link;
    int m_num_nb;
    double m_sigma;
    SegFormat m_format = LabelISPFormat;
    int m_target = 1;
    int levels = 0;
    detail::Buf img;
};
} // namespace hbp_isp

#ifndef HBP_ISP_NO_GLOBAL_NAMES
using hbp_isp::CentoridLink;
using hbp_isp::MaxLink;
using hbp_isp::MinLink;
using hbp_isp::WardLink;
using hbp_isp::BoundaryFormat;
using hbp_isp::EmptyFormat;
using hbp_isp::LabelDeviceIntFormat;
using hbp_isp::LabelIntFormat;
using hbp_isp::LabelISPFormat;
using hbp_isp::LabelUchar3Format;
using hbp_isp::Linkage;
using hbp_isp::SegFormat;
using hbp_isp::SegHAC;
#endif
