// SegHAC with the reference's interface (segment.hpp:8-27, :248): the image
// segmentation pyramid on the B200 engine (hbp_segment_d). The path's
// configuration is offered: CentoridLink (the reference's spelling), 4
// neighbours, sigma 0, LabelISPFormat, target 1; others are rejected. Each
// SegHAC owns the engine context that holds its pyramid; ISPData shares it.
#pragma once

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
        : width(src.cols), height(src.rows)
    {
        detail::need_bgr(src, "SegHAC");
        if (link != CentoridLink || num_nb != 4 || sigma != 0.0 || seg_format != LabelISPFormat ||
            target_clus != 1 || show_cycle)
            throw std::invalid_argument("SegHAC: offered for CentoridLink, 4 neighbours, sigma 0, "
                                        "LabelISPFormat, target 1, no cycle display");
        img = detail::upload(src);
        ctx = std::make_shared<detail::Ctx>();
    }

    // run_ms (segment.cu:1279-1321); per-level images are not produced
    void run_ms(std::vector<Mat> *segs = nullptr)
    {
        if (segs)
            throw std::invalid_argument("SegHAC: per-level label images are not produced");
        detail::check(hbp_segment_d(ctx->h, img->as<uint8_t>(), width, height, &levels, nullptr));
    }

    int g_width() const { return width; }
    int g_height() const { return height; }
    int g_levels() const { return levels; }

    detail::CtxPtr ctx; // holds the pyramid after run_ms

  private:
    int width, height;
    int levels = 0;
    detail::Buf img;
};
} // namespace hbp_isp

#ifndef HBP_ISP_NO_GLOBAL_NAMES
using hbp_isp::CentoridLink;
using hbp_isp::LabelISPFormat;
using hbp_isp::Linkage;
using hbp_isp::SegFormat;
using hbp_isp::SegHAC;
#endif
