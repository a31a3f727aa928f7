// SegHAC with the reference's interface (segment.hpp:8-27, :248): the image
// segmentation pyramid on the B200 engine (hbp_segment_cfg_d). Offered: every
// linkage (CentoridLink is the reference's spelling), 4 or 8 neighbours,
// sigma with round(3 sigma) <= 7, LabelISPFormat, target 1; other formats,
// superpixel targets and cycle display are rejected. Each SegHAC owns the
// engine context that holds its pyramid; ISPData shares it.
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
        if (seg_format != LabelISPFormat || target_clus != 1 || show_cycle)
            throw std::invalid_argument("SegHAC: offered for LabelISPFormat, target 1, no cycle display");
        if (link < MinLink || link > WardLink || (num_nb != 4 && num_nb != 8) || !(sigma >= 0.0) ||
            (int)std::round(3 * sigma) > 7)
            throw std::invalid_argument("SegHAC: linkage Min/Max/Centroid/Ward, 4 or 8 neighbours, "
                                        "round(3 sigma) <= 7");
        img = detail::upload(src);
        ctx = std::make_shared<detail::Ctx>();
    }

    // run_ms (segment.cu:1279-1321); per-level images are not produced
    void run_ms(std::vector<Mat> *segs = nullptr)
    {
        if (segs)
            throw std::invalid_argument("SegHAC: per-level label images are not produced");
        detail::check(hbp_segment_cfg_d(ctx->h, img->as<uint8_t>(), width, height, (int)m_link, m_num_nb, m_sigma,
                                        &levels, nullptr));
    }

    int g_width() const { return width; }
    int g_height() const { return height; }
    int g_levels() const { return levels; }

    detail::CtxPtr ctx; // holds the pyramid after run_ms

  private:
    int width, height;
    Linkage m_link;
    int m_num_nb;
    double m_sigma;
    int levels = 0;
    detail::Buf img;
};
} // namespace hbp_isp

#ifndef HBP_ISP_NO_GLOBAL_NAMES
using hbp_isp::CentoridLink;
using hbp_isp::MaxLink;
using hbp_isp::MinLink;
using hbp_isp::WardLink;
using hbp_isp::LabelISPFormat;
using hbp_isp::Linkage;
using hbp_isp::SegFormat;
using hbp_isp::SegHAC;
#endif
