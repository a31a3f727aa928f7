// PFM disparity files and bad-pixel rates with the reference's interface
// (cvutils.hpp:23-144 cvutils::io::read_pfm_file / save_pfm_file,
// Evaluator.h:6-101), for Middlebury-style reporting, on hbp_isp::Mat.
// The writer stores full rows of 3-channel images (the reference writes only
// `width` floats per row there, cvutils.hpp:135).
#pragma once

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "common.hpp"

namespace hbp_isp
{
namespace cvutils
{
namespace io
{
// read_pfm_file: "Pf" (1 channel) or "PF" (3), width height, scale (negative
// = little endian), then rows bottom-up. The samples are the last
// w*h*channels floats of the file. Returns an empty Mat on any failure.
inline Mat read_pfm_file(const std::string &filename)
{
    FILE *f = std::fopen(filename.c_str(), "rb");
    if (!f)
        return Mat();
    char tag[8] = {0};
    int w = 0, h = 0;
    double scale = 1.0;
    if (std::fscanf(f, "%7s %d %d %lf", tag, &w, &h, &scale) != 4 || w <= 0 || h <= 0)
    {
        std::fclose(f);
        return Mat();
    }
    const int ch = std::strcmp(tag, "Pf") == 0 ? 1 : std::strcmp(tag, "PF") == 0 ? 3 : 0;
    if (ch == 0)
    {
        std::fclose(f);
        return Mat();
    }
    const size_t n = (size_t)w * h * ch;
    std::vector<uint8_t> raw(n * 4);
    if (std::fseek(f, -(long)(n * 4), SEEK_END) != 0 || std::fread(raw.data(), 4, n, f) != n)
    {
        std::fclose(f);
        return Mat();
    }
    std::fclose(f);
    const uint16_t probe = 1;
    const bool native_little = *reinterpret_cast<const uint8_t *>(&probe) == 1;
    const bool file_little = scale < 0.0;
    Mat image(h, w, ch == 1 ? MAT_32FC1 : MAT_32FC3);
    for (size_t i = 0; i < n; ++i)
    {
        uint8_t *p = &raw[4 * i];
        if (file_little != native_little)
        {
            std::swap(p[0], p[3]);
            std::swap(p[1], p[2]);
        }
        const size_t px = i / ch, c = i % ch;
        const size_t row = (size_t)h - 1 - px / (size_t)w, col = px % (size_t)w;
        std::memcpy(image.ptr<float>((int)row) + col * ch + c, p, 4);
    }
    return image;
}

// save_pfm_file: little endian, scale -1/255 as the reference writes it.
inline bool save_pfm_file(const std::string &filename, const Mat &image)
{
    const int ch = image.channels();
    if ((image.type() != MAT_32FC1 && image.type() != MAT_32FC3) || image.empty())
        return false;
    FILE *f = std::fopen(filename.c_str(), "wb");
    if (!f)
        return false;
    std::fprintf(f, "%s\n%d %d\n%lf\n", ch == 1 ? "Pf" : "PF", image.cols, image.rows, -1.0 / 255.0);
    const size_t line = (size_t)image.cols * ch;
    bool ok = true;
    for (int y = image.rows - 1; y >= 0 && ok; --y)
        ok = std::fwrite(image.ptr<float>(y), sizeof(float), line, f) == line;
    std::fclose(f);
    return ok;
}
} // namespace io
} // namespace cvutils

// Evaluator: bad-pixel rates (in %) of a disparity map against ground truth,
// over all valid pixels (ground truth > 0 and finite), the non-occluded mask
// and the occluded rest; a pixel is bad when |d - gt| > the threshold
// (default 0.5). nonocc_mask: MAT_8UC1, non-zero = non-occluded. The
// reference's image and log outputs are left out.
class Evaluator
{
  public:
    struct Rates
    {
        double all, nonocc, occ;
    };

    Evaluator(const Mat &dispGT, const Mat &nonoccMask) : gt(dispGT), nonocc(nonoccMask)
    {
        if (gt.type() != MAT_32FC1 || nonocc.type() != MAT_8UC1 || gt.rows != nonocc.rows || gt.cols != nonocc.cols)
            throw std::invalid_argument("Evaluator: float ground truth and uint8 mask of one size");
    }
    void setErrorThreshold(double t) { threshold = t; }

    Rates evaluate(const Mat &disp) const
    {
        if (disp.type() != MAT_32FC1 || disp.rows != gt.rows || disp.cols != gt.cols)
            throw std::invalid_argument("Evaluator: disparity of the ground truth's size expected");
        long valid = 0, non = 0, occ = 0, good_valid = 0, good_non = 0, good_occ = 0;
        const size_t n = gt.total();
        const float *g = gt.ptr<float>(), *d = disp.ptr<float>();
        const uint8_t *m = nonocc.ptr<uint8_t>();
        for (size_t i = 0; i < n; ++i)
        {
            const bool v = g[i] > 0.0f && g[i] != INFINITY;
            const bool good = std::fabs(d[i] - g[i]) <= threshold;
            const bool nn = m[i] != 0;
            valid += v;
            good_valid += v && good;
            non += nn;
            good_non += nn && good;
            occ += v && !nn;
            good_occ += v && !nn && good;
        }
        auto rate = [](long good, long total) { return total ? 100.0 * (1.0 - (double)good / total) : 0.0; };
        return {rate(good_valid, valid), rate(good_non, non), rate(good_occ, occ)};
    }

  private:
    Mat gt, nonocc;
    double threshold = 0.5;
};
} // namespace hbp_isp

#ifndef HBP_ISP_NO_GLOBAL_NAMES
namespace cvutils = hbp_isp::cvutils;
using hbp_isp::Evaluator;
#endif
