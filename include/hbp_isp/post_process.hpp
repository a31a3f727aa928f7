// PostProcess with the reference's interface (post_process.hpp:8-61) and the
// single-pair driver's medianFilter (main_stereo_hbp_isp.cu:120-192), on the
// B200 engine. As in the reference, the LR check fills and the median filters
// the left view only; median_filter uses the failure mask of the last
// left_right_check.
#pragma once

#include "common.hpp"

namespace hbp_isp
{
class PostProcess
{
  public:
    PostProcess(const Mat &imL, const Mat &imR) : width(imL.cols), height(imL.rows)
    {
        detail::need_bgr(imL, "PostProcess");
        detail::need_bgr(imR, "PostProcess");
        left = detail::upload(imL);
    }

    using Result = std::pair<Mat, Mat>;

    // left_right_check (post_process.cu:47-110)
    void left_right_check(Result &results_left, Result &results_right)
    {
        detail::Buf dL = detail::upload(results_left.first), dR = detail::upload(results_right.first);
        detail::Buf pL = detail::upload(results_left.second);
        fail = std::make_shared<detail::DevBuf>((size_t)width * height);
        detail::check(hbp_lr_check_d(detail::shared_ctx()->h, dL->as<float>(), dR->as<float>(), pL->as<float>(),
                                     fail->as<uint8_t>(), nullptr, width, height, nullptr));
        detail::download(results_left.second, pL);
    }

    // median_filter (post_process.cu:112-185)
    void median_filter(Result &results_left, Result &)
    {
        if (!fail)
            throw std::logic_error("PostProcess: left_right_check() comes before median_filter()");
        detail::Buf pL = detail::upload(results_left.second);
        detail::check(hbp_weighted_median_d(detail::shared_ctx()->h, left->as<uint8_t>(), fail->as<uint8_t>(),
                                            pL->as<float>(), nullptr, width, height, nullptr));
        detail::download(results_left.second, pL);
    }
    // median_filter_gpu (post_process.cu:245-371): the reference's GPU variant
    // (device expf weights, float sums, bubble-sort tie order)
    void median_filter_gpu(Result &results_left, Result &)
    {
        if (!fail)
            throw std::logic_error("PostProcess: left_right_check() comes before median_filter_gpu()");
        detail::Buf pL = detail::upload(results_left.second);
        detail::check(hbp_weighted_median_gpu_d(detail::shared_ctx()->h, left->as<uint8_t>(), fail->as<uint8_t>(),
                                                pL->as<float>(), nullptr, width, height, nullptr));
        detail::download(results_left.second, pL);
    }

    // plane_label_to_disp (post_process.cu:373-390)
    void plane_label_to_disp(Result &results_left, Result &)
    {
        detail::Buf pL = detail::upload(results_left.second);
        detail::Buf d = std::make_shared<detail::DevBuf>(4 * (size_t)width * height);
        detail::check(hbp_plane_to_disp_d(detail::shared_ctx()->h, pL->as<float>(), d->as<float>(), width, height,
                                          nullptr));
        detail::download(results_left.first, d);
    }

  private:
    int width, height;
    detail::Buf left, fail;
};

// medianFilter of the single-pair driver: 7-tap horizontal then vertical
// median of a MAT_32FC1 disparity, in place
inline void medianFilter(Mat &D)
{
    detail::Buf d = detail::upload(D);
    detail::check(hbp_driver_median_d(detail::shared_ctx()->h, d->as<float>(), D.cols, D.rows, nullptr));
    detail::download(D, d);
}
} // namespace hbp_isp

#ifndef HBP_ISP_NO_GLOBAL_NAMES
using hbp_isp::medianFilter;
using hbp_isp::PostProcess;
#endif
