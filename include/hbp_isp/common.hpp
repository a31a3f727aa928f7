// C++ classes with the interface of the reference's stereo path (StereoCost,
// CRTrees, SegHAC, ISPData, StereoData, HBP_ISP, PostProcess, medianFilter),
// header-only, on top of the C ABI of libhbp_b200.so (include/hbp_b200.h).
// This file: the image type standing in for cv::Mat, device buffers and
// contexts, error handling. Where <opencv2/core.hpp> is on the include path,
// hbp_isp::Mat converts from and to cv::Mat, so the reference's call sites
// can pass and receive cv::Mat.
#pragma once

#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../hbp_b200.h"

#if __has_include(<opencv2/core.hpp>)
#include <opencv2/core.hpp>
#define HBP_ISP_WITH_OPENCV 1
#endif

namespace hbp_isp
{

// Element types, with OpenCV's codes (CV_8UC1, CV_8UC3, CV_32SC1, CV_32FC1,
// CV_32FC3).
enum MatType
{
    MAT_8UC1 = 0,
    MAT_8UC3 = 16,
    MAT_32SC1 = 4,
    MAT_32FC1 = 5,
    MAT_32FC3 = 21
};

// A host image: rows x cols x channels of uint8, int32 or float, row-major and
// contiguous (cv::Mat's continuous layout). It owns its pixels, or wraps a
// caller's buffer (a cv::Mat's .data, for instance) without copying.
class Mat
{
  public:
    int rows = 0, cols = 0;
    uint8_t *data = nullptr;

    Mat() = default;
    Mat(int r, int c, int type) : rows(r), cols(c), type_(type)
    {
        own_ = std::make_shared<std::vector<uint8_t>>(bytes(), 0);
        data = own_->data();
    }
    Mat(int r, int c, int type, void *external) : rows(r), cols(c), data(static_cast<uint8_t *>(external)), type_(type) {}
#ifdef HBP_ISP_WITH_OPENCV
    // a cv::Mat's pixels, wrapped without copying (the cv::Mat keeps them):
    // continuous and of one of the types above
    Mat(const cv::Mat &m) : rows(m.rows), cols(m.cols), data(static_cast<uint8_t *>(m.data)), type_(m.type())
    {
        const bool known = type_ == MAT_8UC1 || type_ == MAT_8UC3 || type_ == MAT_32SC1 || type_ == MAT_32FC1 ||
                           type_ == MAT_32FC3;
        if (!m.empty() && (!known || !m.isContinuous()))
            throw std::invalid_argument("hbp_isp::Mat: a continuous cv::Mat of type CV_8UC1, CV_8UC3, CV_32SC1, "
                                        "CV_32FC1 or CV_32FC3 is required");
    }
    // a cv::Mat holding a copy of these pixels
    operator cv::Mat() const { return empty() ? cv::Mat() : cv::Mat(rows, cols, type_, data).clone(); }
#endif

    int type() const { return type_; }
    int channels() const { return type_ == MAT_8UC3 || type_ == MAT_32FC3 ? 3 : 1; }
    size_t elemSize1() const { return type_ == MAT_32FC1 || type_ == MAT_32FC3 || type_ == MAT_32SC1 ? 4 : 1; }
    size_t elemSize() const { return elemSize1() * (size_t)channels(); }
    size_t total() const { return (size_t)rows * (size_t)cols; }
    size_t bytes() const { return total() * elemSize(); }
    bool empty() const { return data == nullptr || total() == 0; }
    Mat clone() const
    {
        Mat m(rows, cols, type_);
        if (bytes())
            std::memcpy(m.data, data, bytes());
        return m;
    }
    template <typename T>
    T *ptr(int r = 0)
    {
        return reinterpret_cast<T *>(data + (size_t)r * cols * elemSize());
    }
    template <typename T>
    const T *ptr(int r = 0) const
    {
        return reinterpret_cast<const T *>(data + (size_t)r * cols * elemSize());
    }
    template <typename T>
    T &at(int r, int c)
    {
        return ptr<T>(r)[c];
    }

  private:
    int type_ = MAT_8UC1;
    std::shared_ptr<std::vector<uint8_t>> own_;
};

namespace detail
{
inline void check(hbp_status s)
{
    if (s != HBP_OK)
        throw std::runtime_error(std::string("hbp_b200: ") + hbp_status_string(s) + ": " + hbp_last_error());
}

// Device memory of the engine's device 0 (the reference runs on the current
// device with the legacy stream; so do these classes).
struct DevBuf
{
    void *p = nullptr;
    size_t n = 0;
    explicit DevBuf(size_t bytes) : n(bytes) { check(hbp_dev_alloc(0, bytes, &p)); }
    ~DevBuf() { hbp_dev_free(p); }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    template <typename T>
    T *as() const
    {
        return static_cast<T *>(p);
    }
};
using Buf = std::shared_ptr<DevBuf>;

inline Buf upload(const Mat &m)
{
    Buf b = std::make_shared<DevBuf>(m.bytes());
    check(hbp_copy(b->p, m.data, m.bytes()));
    return b;
}

inline void download(Mat &m, const Buf &b) { check(hbp_copy(m.data, b->p, m.bytes())); }

// An engine context (device 0): its scratch, and the pyramid of a SegHAC.
struct Ctx
{
    hbp_ctx *h = nullptr;
    Ctx() { check(hbp_ctx_create(0, 0, 0, &h)); }
    ~Ctx() { hbp_ctx_destroy(h); }
    Ctx(const Ctx &) = delete;
    Ctx &operator=(const Ctx &) = delete;
};
using CtxPtr = std::shared_ptr<Ctx>;

// The context of the stages that keep nothing between calls.
inline const CtxPtr &shared_ctx()
{
    static CtxPtr c = std::make_shared<Ctx>();
    return c;
}

inline void need_bgr(const Mat &m, const char *who)
{
    if (m.type() != MAT_8UC3 || m.empty())
        throw std::invalid_argument(std::string(who) + ": a BGR8 image (3 channels of uint8) is required");
}
} // namespace detail
} // namespace hbp_isp
