// Minimal stand-in for the parts of OpenCV's C++ API that the reference sources
// (stereo_cost.hpp/.cu, segment.hpp/.cu, hbp_isp.hpp/.cu, post_process.hpp/.cu,
// cvutils.hpp) name. It exists only so that the reference's own CUDA/C++ files
// compile unmodified into the checker library oracle/_ref/libhbpref.so; the
// container has no OpenCV C++ headers or libraries.
//
// Implemented for real (the reference's data path runs through them):
//   Mat (2-D and 3-D, 8U/32S/32F with 1-4 channels, ROI headers, clone, copyTo,
//   convertTo, at<>, ptr<>, zeros, comparison with a scalar), Mat_<T>, Rect,
//   Point, Size, Vec, Scalar, dilate (3x3 box, out-of-image samples ignored, as
//   OpenCV's default dilate border does).
// Declared only so that unused inline helpers in cvutils.hpp parse (calling
// them aborts): reduce, boxFilter, merge, resize, sqrt, theRNG, cvtColor,
// circle, line, Mat::mul/reshape.
#pragma once

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

typedef unsigned char uchar;

#define CV_8U 0
#define CV_8S 1
#define CV_16U 2
#define CV_16S 3
#define CV_32S 4
#define CV_32F 5
#define CV_64F 6
#define CV_CN_SHIFT 3
#define CV_DEPTH_MASK 7
#define CV_MAKETYPE(depth, cn) ((depth) + (((cn) - 1) << CV_CN_SHIFT))
#define CV_MAKE_TYPE CV_MAKETYPE
#define CV_MAT_DEPTH(t) ((t) & CV_DEPTH_MASK)
#define CV_MAT_CN(t) ((((t) >> CV_CN_SHIFT) & 63) + 1)
#define CV_8UC1 CV_MAKETYPE(CV_8U, 1)
#define CV_8UC3 CV_MAKETYPE(CV_8U, 3)
#define CV_32SC1 CV_MAKETYPE(CV_32S, 1)
#define CV_32FC1 CV_MAKETYPE(CV_32F, 1)
#define CV_32FC3 CV_MAKETYPE(CV_32F, 3)
#ifndef CV_PI
#define CV_PI 3.1415926535897932384626433832795
#endif

namespace cv
{
[[noreturn]] inline void shim_unsupported(const char *what)
{
    std::fprintf(stderr, "cvshim: %s is not provided by the shim\n", what);
    std::abort();
}

struct Size
{
    int width = 0, height = 0;
    Size() {}
    Size(int w, int h) : width(w), height(h) {}
    int area() const { return width * height; }
    bool operator==(const Size &o) const { return width == o.width && height == o.height; }
};

template <typename T>
struct Point_
{
    T x = 0, y = 0;
    Point_() {}
    Point_(T x_, T y_) : x(x_), y(y_) {}
};
typedef Point_<int> Point;
typedef Point_<float> Point2f;

struct Rect
{
    int x = 0, y = 0, width = 0, height = 0;
    Rect() {}
    Rect(int x_, int y_, int w, int h) : x(x_), y(y_), width(w), height(h) {}
    Rect(const Point &p, const Size &s) : x(p.x), y(p.y), width(s.width), height(s.height) {}
    Point br() const { return Point(x + width, y + height); }
    bool contains(const Point &p) const
    {
        return x <= p.x && p.x < x + width && y <= p.y && p.y < y + height;
    }
    Rect operator&(const Rect &o) const
    {
        int x0 = std::max(x, o.x), y0 = std::max(y, o.y);
        int x1 = std::min(x + width, o.x + o.width), y1 = std::min(y + height, o.y + o.height);
        if (x1 <= x0 || y1 <= y0)
            return Rect();
        return Rect(x0, y0, x1 - x0, y1 - y0);
    }
};

template <typename T, int n>
struct Vec
{
    T val[n];
    Vec() { for (int i = 0; i < n; ++i) val[i] = T(0); }
    Vec(T a, T b, T c) { static_assert(n == 3, "3-vector"); val[0] = a; val[1] = b; val[2] = c; }
    T &operator[](int i) { return val[i]; }
    const T &operator[](int i) const { return val[i]; }
    Vec operator-(const Vec &o) const
    {
        Vec r;
        for (int i = 0; i < n; ++i) r.val[i] = val[i] - o.val[i];
        return r;
    }
};
typedef Vec<float, 3> Vec3f;
typedef Vec<double, 3> Vec3d;

struct Scalar
{
    double val[4];
    Scalar(double a = 0, double b = 0, double c = 0, double d = 0)
    {
        val[0] = a; val[1] = b; val[2] = c; val[3] = d;
    }
    static Scalar all(double v) { return Scalar(v, v, v, v); }
};

inline size_t shim_depth_size(int depth)
{
    switch (depth)
    {
    case CV_8U: case CV_8S: return 1;
    case CV_16U: case CV_16S: return 2;
    case CV_32S: case CV_32F: return 4;
    case CV_64F: return 8;
    }
    return 1;
}

class Mat
{
public:
    struct MSize
    {
        const Mat *m;
        const int *p;
        int operator[](int i) const { return p[i]; }
        Size operator()() const { return Size(m->cols, m->rows); }
    };

    int flags_type = 0;
    int dims = 0;
    int rows = 0, cols = 0;
    uchar *data = nullptr;
    size_t step = 0; // bytes between rows (2-D)
    int sizes_[3] = {0, 0, 0};
    MSize size;
    std::shared_ptr<std::vector<uchar>> buf;

    Mat() { size = MSize{this, sizes_}; }
    Mat(int r, int c, int type) : Mat() { create(r, c, type); }
    Mat(int r, int c, int type, const Scalar &s) : Mat() { create(r, c, type); setTo(s); }
    Mat(Size sz, int type) : Mat() { create(sz.height, sz.width, type); }
    Mat(int ndims, const int *szs, int type) : Mat() { create(ndims, szs, type); }
    Mat(int r, int c, int type, void *ext) : Mat()
    {
        flags_type = type; dims = 2; rows = r; cols = c;
        sizes_[0] = r; sizes_[1] = c;
        step = (size_t)c * elemSize();
        data = (uchar *)ext;
    }
    Mat(const Mat &o) { *this = o; }
    Mat &operator=(const Mat &o)
    {
        flags_type = o.flags_type; dims = o.dims; rows = o.rows; cols = o.cols;
        data = o.data; step = o.step; buf = o.buf;
        std::memcpy(sizes_, o.sizes_, sizeof(sizes_));
        size = MSize{this, sizes_};
        return *this;
    }

    int type() const { return flags_type; }
    int depth() const { return CV_MAT_DEPTH(flags_type); }
    int channels() const { return CV_MAT_CN(flags_type); }
    size_t elemSize() const { return shim_depth_size(depth()) * channels(); }
    size_t total() const
    {
        size_t t = 1;
        for (int i = 0; i < dims; ++i) t *= (size_t)sizes_[i];
        return dims ? t : 0;
    }
    bool empty() const { return data == nullptr || total() == 0; }
    bool isContinuous() const { return dims != 2 || step == (size_t)cols * elemSize(); }

    void create(int r, int c, int type)
    {
        int szs[2] = {r, c};
        create(2, szs, type);
    }
    void create(int ndims, const int *szs, int type)
    {
        flags_type = type; dims = ndims;
        for (int i = 0; i < 3; ++i) sizes_[i] = i < ndims ? szs[i] : 0;
        rows = ndims >= 1 ? szs[0] : 0;
        cols = ndims >= 2 ? szs[1] : 0;
        if (ndims == 3) { rows = -1; cols = -1; }
        size_t n = 1;
        for (int i = 0; i < ndims; ++i) n *= (size_t)szs[i];
        buf = std::make_shared<std::vector<uchar>>(n * elemSize(), (uchar)0);
        data = buf->data();
        step = ndims == 2 ? (size_t)szs[1] * elemSize() : 0;
        size = MSize{this, sizes_};
    }
    void release() { buf.reset(); data = nullptr; dims = rows = cols = 0; }

    void setTo(const Scalar &s)
    {
        int cn = channels();
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < cols; ++c)
                for (int k = 0; k < cn; ++k)
                    set_elem(r, c, k, s.val[k < 4 ? k : 3]);
    }

    template <typename T> T *ptr(int r = 0) { return (T *)(data + (size_t)r * step); }
    template <typename T> const T *ptr(int r = 0) const { return (const T *)(data + (size_t)r * step); }
    template <typename T> T *ptr(int i0, int i1)
    {
        // 3-D continuous volume: plane i0, row i1
        return (T *)(data + ((size_t)i0 * sizes_[1] + i1) * sizes_[2] * elemSize());
    }
    template <typename T> T &at(int r, int c) { return ((T *)(data + (size_t)r * step))[c]; }
    template <typename T> const T &at(int r, int c) const { return ((const T *)(data + (size_t)r * step))[c]; }
    template <typename T> T &at(const Point &p) { return at<T>(p.y, p.x); }
    template <typename T> const T &at(const Point &p) const { return at<T>(p.y, p.x); }

    Mat clone() const
    {
        Mat m;
        if (dims == 3)
        {
            m.create(3, sizes_, flags_type);
            std::memcpy(m.data, data, total() * elemSize());
            return m;
        }
        m.create(rows, cols, flags_type);
        for (int r = 0; r < rows; ++r)
            std::memcpy(m.ptr<uchar>(r), ptr<uchar>(r), (size_t)cols * elemSize());
        return m;
    }
    // Copy into an existing header of the same shape (ROI or full image).
    void copy_into(const Mat &dst) const
    {
        for (int r = 0; r < rows; ++r)
            std::memcpy(dst.data + (size_t)r * dst.step, ptr<uchar>(r), (size_t)cols * elemSize());
    }
    void copyTo(Mat &&dst) const
    {
        if (dst.data && dst.rows == rows && dst.cols == cols && dst.flags_type == flags_type)
            return copy_into(dst);
        shim_unsupported("Mat::copyTo into a differently shaped header");
    }
    void copyTo(Mat &dst) const
    {
        if (dst.data && dst.rows == rows && dst.cols == cols && dst.flags_type == flags_type)
            return copy_into(dst);
        dst = clone();
    }
    Mat operator()(const Rect &r) const
    {
        Mat m(*this);
        m.data = data + (size_t)r.y * step + (size_t)r.x * elemSize();
        m.rows = r.height; m.cols = r.width;
        m.sizes_[0] = r.height; m.sizes_[1] = r.width;
        return m;
    }
    Mat col(int c) const { return (*this)(Rect(c, 0, 1, rows)); }

    double get_elem(int r, int c, int k) const
    {
        const uchar *p = data + (size_t)r * step + (size_t)c * elemSize() + k * shim_depth_size(depth());
        switch (depth())
        {
        case CV_8U: return *p;
        case CV_32S: return *(const int *)p;
        case CV_32F: return *(const float *)p;
        case CV_64F: return *(const double *)p;
        }
        shim_unsupported("element depth");
    }
    void set_elem(int r, int c, int k, double v)
    {
        uchar *p = data + (size_t)r * step + (size_t)c * elemSize() + k * shim_depth_size(depth());
        switch (depth())
        {
        case CV_8U: *p = (uchar)std::min(255.0, std::max(0.0, std::nearbyint(v))); return;
        case CV_32S: *(int *)p = (int)std::nearbyint(v); return;
        case CV_32F: *(float *)p = (float)v; return;
        case CV_64F: *(double *)p = v; return;
        }
        shim_unsupported("element depth");
    }
    // OpenCV semantics: dst = saturate_cast<depth>(src * alpha + beta), channels kept.
    void convertTo(Mat &dst, int rtype, double alpha = 1.0, double beta = 0.0) const
    {
        int ddepth = rtype < 0 ? depth() : CV_MAT_DEPTH(rtype);
        Mat out(rows, cols, CV_MAKETYPE(ddepth, channels()));
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < cols; ++c)
                for (int k = 0; k < channels(); ++k)
                {
                    double v = get_elem(r, c, k);
                    if (alpha != 1.0 || beta != 0.0)
                        v = v * alpha + beta;
                    out.set_elem(r, c, k, v);
                }
        dst = out;
    }

    static Mat zeros(Size sz, int type) { return Mat(sz, type); }
    static Mat zeros(int r, int c, int type) { return Mat(r, c, type); }

    Mat mul(const Mat &, double = 1) const { shim_unsupported("Mat::mul"); }
    Mat mul(const Scalar &) const { shim_unsupported("Mat::mul"); }
    Mat reshape(int, int = 0) const { shim_unsupported("Mat::reshape"); }
};

// Element-wise comparison with a scalar: 255 where true, 0 elsewhere (CV_8U).
inline Mat operator>(const Mat &a, double s)
{
    Mat out(a.rows, a.cols, CV_8UC1);
    for (int r = 0; r < a.rows; ++r)
        for (int c = 0; c < a.cols; ++c)
            out.at<uchar>(r, c) = a.get_elem(r, c, 0) > s ? 255 : 0;
    return out;
}
inline Mat operator-(const Mat &, const Mat &) { shim_unsupported("Mat subtraction"); }

template <typename T>
class Mat_ : public Mat
{
public:
    Mat_() : Mat() {}
    Mat_(int ndims, const int *szs) : Mat(ndims, szs, type_of()) {}
    Mat_(int r, int c, T *ext) : Mat(r, c, type_of(), (void *)ext) {}
    Mat_(Size sz, T v) : Mat(sz, type_of()) { setTo(Scalar::all((double)v)); }
    Mat_(const Mat &m) : Mat(m) {}
    Mat_ operator()(const Rect &r) const { return Mat_(Mat::operator()(r)); }
    static int type_of()
    {
        if (sizeof(T) == 1) return CV_8UC1;
        if (sizeof(T) == 4 && T(0.5) != T(0)) return CV_32FC1;
        return CV_32SC1;
    }
};

// 3x3 rectangular dilation of an 8-bit single-channel image. Samples outside
// the image do not take part (OpenCV's default border value for dilate).
inline void dilate(const Mat &src, Mat &dst, const Mat & /*kernel: 3x3 default*/)
{
    Mat out(src.rows, src.cols, CV_8UC1);
    for (int r = 0; r < src.rows; ++r)
        for (int c = 0; c < src.cols; ++c)
        {
            uchar m = 0;
            for (int dr = -1; dr <= 1; ++dr)
                for (int dc = -1; dc <= 1; ++dc)
                {
                    int rr = r + dr, cc = c + dc;
                    if (rr < 0 || cc < 0 || rr >= src.rows || cc >= src.cols)
                        continue;
                    m = std::max(m, src.at<uchar>(rr, cc));
                }
            out.at<uchar>(r, c) = m;
        }
    dst = out;
}

enum { COLOR_Lab2BGR = 57, LINE_AA = 16, REDUCE_SUM = 0, BORDER_CONSTANT = 0, INTER_LINEAR = 1, INTER_NEAREST = 0, IMREAD_COLOR = 1, IMREAD_GRAYSCALE = 0 };

inline void cvtColor(const Mat &, Mat &, int) { shim_unsupported("cvtColor"); }
inline void circle(Mat &, Point2f, int, const Scalar &, int = 1, int = 8) { shim_unsupported("circle"); }
inline void line(Mat &, Point2f, Point2f, const Scalar &, int = 1, int = 8) { shim_unsupported("line"); }
inline void reduce(const Mat &, Mat &, int, int) { shim_unsupported("reduce"); }
inline void boxFilter(const Mat &, Mat &, int, Size, Point, bool, int) { shim_unsupported("boxFilter"); }
inline void merge(const std::vector<Mat> &, Mat &) { shim_unsupported("merge"); }
inline void resize(const Mat &, Mat &, Size, double = 0, double = 0, int = 1) { shim_unsupported("resize"); }
inline void sqrt(const Mat &, Mat &) { shim_unsupported("sqrt"); }
struct RNG
{
    double uniform(double, double) { shim_unsupported("RNG"); }
};
inline RNG &theRNG()
{
    static RNG r;
    return r;
}
typedef std::string String;
} // namespace cv
