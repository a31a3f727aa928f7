// ISPData, StereoData and HBP_ISP with the reference's interface
// (hbp_isp.hpp:9-126, :288): hierarchical BP on the segmentation pyramid on
// the B200 engine (hbp_infer_d; hbp_infer_f32_d on an MC-CNN volume). ISPData shares its SegHAC's pyramid and
// StereoData its StereoCost's volume (the reference deep-copies both), so
// either producer may be deleted first, as the reference's drivers do.
// Extension: set_msg_fp16() stores the BP messages as FP16.
#pragma once

#include <tuple>

#include "segment.hpp"
#include "stereo_cost.hpp"

namespace hbp_isp
{
class ISPData
{
  public:
    explicit ISPData(const SegHAC *const seg) : width(seg->g_width()), height(seg->g_height()), ctx(seg->ctx)
    {
        if (seg->g_levels() <= 0)
            throw std::invalid_argument("ISPData: run_ms() the SegHAC first");
        std::vector<int> sizes(2 * 64);
        detail::check(hbp_pyramid_levels(ctx->h, sizes.data(), 64));
        for (int l = 0; l < 64 && sizes[2 * l] > 0; ++l)
        {
            num_clus_isp.push_back(sizes[2 * l]);
            num_bd_isp.push_back(sizes[2 * l + 1]);
        }
    }
    int g_width() const { return width; }
    int g_height() const { return height; }
    int g_mean_channels() const { return 6; }
    std::vector<int> g_num_clus_isp() const { return num_clus_isp; }
    std::vector<int> g_num_bd_isp() const { return num_bd_isp; }
    // the ISP arrays in place on the device (hbp_isp.hpp:18-21; bd as int
    // pairs); they belong to the SegHAC's context, so a later run_ms of that
    // SegHAC replaces them (the reference's ISPData holds a copy)
    const int *g_isp_clus_d() const { return device_arrays(0).c; }
    const float *g_isp_mean_d() const { return device_arrays(1).m; }
    const int *g_isp_bd_d() const { return device_arrays(2).c; }
    const int *g_isp_bdl_d() const { return device_arrays(3).c; }
    // the same on the host: clus, mean sums [6][N_l], bd pairs, bdl,
    // concatenated over levels
    void copy_isp(std::vector<int> &clus, std::vector<float> &mean, std::vector<int> &bd,
                  std::vector<int> &bdl) const
    {
        size_t tn = 0, te = 0;
        for (size_t l = 0; l < num_clus_isp.size(); ++l)
        {
            tn += (size_t)num_clus_isp[l];
            te += (size_t)num_bd_isp[l];
        }
        clus.resize(tn);
        mean.resize(6 * tn);
        bd.resize(2 * te);
        bdl.resize(te);
        detail::check(hbp_pyramid_copy(ctx->h, clus.data(), mean.data(), bd.data(), bdl.data()));
    }

    int width, height;
    detail::CtxPtr ctx;
    std::vector<int> num_clus_isp, num_bd_isp;

  private:
    struct Ptr
    {
        const int *c = nullptr;
        const float *m = nullptr;
    };
    Ptr device_arrays(int which) const
    {
        const int *clus = nullptr, *bd = nullptr, *bdl = nullptr;
        const float *mean = nullptr;
        detail::check(hbp_pyramid_device(ctx->h, &clus, &mean, &bd, &bdl));
        Ptr p;
        p.c = which == 0 ? clus : which == 2 ? bd : bdl;
        p.m = mean;
        return p;
    }

  public:
};

class StereoData
{
  public:
    StereoData(const StereoCost *const sc, const bool use_cost_vol)
        : m_labels(sc->g_labels()), im_size(sc->g_im_size()), width(sc->g_width()), height(sc->g_height()),
          use_cost_vol(use_cost_vol), f32(sc->g_is_f32()), m_tau(sc->g_tau()), vol(sc->vol), wta(sc->wta)
    {
        if (!use_cost_vol)
            throw std::invalid_argument("StereoData: the path runs on the cost volume (use_cost_vol = true)");
        if (!vol || !wta)
            throw std::invalid_argument("StereoData: compute_stereo_cost() the StereoCost first");
    }
    int g_labels() const { return m_labels; }
    int g_im_size() const { return im_size; }
    float *g_im_D_d() const { return wta->as<float>(); }
    bool g_use_cost_vol() const { return use_cost_vol; }
    const uint8_t *g_img_cost_d() const { return f32 ? nullptr : vol->as<uint8_t>(); }
    const float *g_img_cost_f32_d() const { return f32 ? vol->as<float>() : nullptr; }
    float g_tau() const { return m_tau; }

    int m_labels, im_size, width, height;
    bool use_cost_vol, f32;
    float m_tau;
    detail::Buf vol, wta;
};

class HBP_ISP
{
  public:
    HBP_ISP(const ISPData *const isp_data, const StereoData *const stereo_data, float alpha, float tau_smooth)
        : isp(isp_data), sd(stereo_data), m_alpha(alpha), m_tau_smooth(tau_smooth)
    {
        if (isp->width != sd->width || isp->height != sd->height)
            throw std::invalid_argument("HBP_ISP: pyramid and cost volume differ in size");
    }

    void set_msg_fp16(bool on) { fp16 = on; }

    // run_ms (hbp_isp.cu:1313-1346): disparity (MAT_32FC1) and plane labels
    // (MAT_32FC3, a b c) of min_level
    std::pair<Mat, Mat> run_ms(const int min_level)
    {
        const size_t n = (size_t)isp->width * isp->height;
        hbp_params p;
        hbp_default_params(&p);
        p.alpha = m_alpha;
        p.tau_smooth = m_tau_smooth;
        p.min_level = min_level;
        p.msg_fp16 = fp16 ? 1 : 0;
        p.post = 0;
        detail::Buf d = std::make_shared<detail::DevBuf>(4 * n), pl = std::make_shared<detail::DevBuf>(12 * n);
        if (sd->f32)
            detail::check(hbp_infer_f32_d(isp->ctx->h, sd->vol->as<float>(), sd->wta->as<float>(), sd->m_labels,
                                          sd->m_tau, &p, d->as<float>(), pl->as<float>(), nullptr));
        else
            detail::check(hbp_infer_d(isp->ctx->h, sd->vol->as<uint8_t>(), sd->wta->as<float>(), sd->m_labels, &p,
                                      d->as<float>(), pl->as<float>(), nullptr));
        Mat disp(isp->height, isp->width, MAT_32FC1), plane(isp->height, isp->width, MAT_32FC3);
        detail::download(disp, d);
        detail::download(plane, pl);
        return {disp, plane};
    }

    // run_ms_vis (hbp_isp.cu:1348-1383): (disparity, planes, superpixel
    // image) of every level from the top level down to min_level. The
    // superpixel image is visualisation (cvtColor, circles, lines) and is
    // left empty here.
    std::vector<std::tuple<Mat, Mat, Mat>> run_ms_vis(const int min_level)
    {
        const size_t n = (size_t)isp->width * isp->height;
        const int levels = (int)isp->g_num_clus_isp().size() - min_level;
        if (min_level < 0 || levels < 1)
            throw std::invalid_argument("HBP_ISP: min_level must lie in [0, levels-1]");
        hbp_params p;
        hbp_default_params(&p);
        p.alpha = m_alpha;
        p.tau_smooth = m_tau_smooth;
        p.min_level = min_level;
        p.msg_fp16 = fp16 ? 1 : 0;
        p.post = 0;
        detail::Buf d = std::make_shared<detail::DevBuf>(4 * n * levels);
        detail::Buf pl = std::make_shared<detail::DevBuf>(12 * n * levels);
        int got = 0;
        detail::check(hbp_infer_levels_d(isp->ctx->h, sd->f32 ? nullptr : sd->vol->as<uint8_t>(),
                                         sd->f32 ? sd->vol->as<float>() : nullptr, sd->wta->as<float>(),
                                         sd->m_labels, sd->m_tau, &p, levels, d->as<float>(), pl->as<float>(), &got,
                                         nullptr));
        std::vector<std::tuple<Mat, Mat, Mat>> out;
        for (int k = 0; k < got; ++k)
        {
            Mat disp(isp->height, isp->width, MAT_32FC1), plane(isp->height, isp->width, MAT_32FC3);
            detail::check(hbp_copy(disp.data, d->as<float>() + k * n, disp.bytes()));
            detail::check(hbp_copy(plane.data, pl->as<float>() + 3 * k * n, plane.bytes()));
            out.emplace_back(disp, plane, Mat());
        }
        return out;
    }

  private:
    const ISPData *isp;
    const StereoData *sd;
    float m_alpha, m_tau_smooth;
    bool fp16 = false;
};
} // namespace hbp_isp

#ifndef HBP_ISP_NO_GLOBAL_NAMES
using hbp_isp::HBP_ISP;
using hbp_isp::ISPData;
using hbp_isp::StereoData;
#endif
