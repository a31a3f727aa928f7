// hbp_isp::Mat from and to cv::Mat (include/hbp_isp/common.hpp), against the
// OpenCV stand-in: wrapping shares the pixels, converting back copies them,
// and a non-continuous or unsupported cv::Mat is refused. Host only.
#include <cstdio>

#include "hbp_isp/common.hpp"

#ifndef HBP_ISP_WITH_OPENCV
#error "the OpenCV stand-in was not found"
#endif

int main()
{
    cv::Mat img(4, 6, CV_8UC3);
    for (size_t i = 0; i < img.total() * img.elemSize(); ++i)
        img.data[i] = (uchar)(i * 7);
    hbp_isp::Mat m = img; // no copy
    if (m.data != img.data || m.rows != 4 || m.cols != 6 || m.type() != hbp_isp::MAT_8UC3)
        return 1;
    cv::Mat back = m; // a copy
    if (back.data == img.data || back.type() != CV_8UC3 || back.rows != 4 || back.cols != 6)
        return 2;
    for (size_t i = 0; i < img.total() * img.elemSize(); ++i)
        if (back.data[i] != img.data[i])
            return 3;
    cv::Mat lab(3, 5, CV_32SC1);
    hbp_isp::Mat ml = lab;
    if (ml.elemSize() != 4 || ml.bytes() != 60)
        return 4;
    try
    {
        cv::Mat d(2, 2, CV_MAKETYPE(CV_64F, 1));
        hbp_isp::Mat md = d;
        (void)md;
        return 5;
    }
    catch (const std::invalid_argument &)
    {
    }
    try
    {
        cv::Mat roi = img(cv::Rect(1, 1, 3, 2)); // rows of a larger image
        hbp_isp::Mat mr = roi;
        (void)mr;
        return 6;
    }
    catch (const std::invalid_argument &)
    {
    }
    std::puts("ok");
    return 0;
}
