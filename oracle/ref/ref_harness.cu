// C-ABI entry points around the reference's own classes and kernels, compiled
// together with the unmodified reference sources into oracle/_ref/libhbpref.so.
// This file is test infrastructure: it lets the parity tests and the golden
// fixture script run the reference implementation on the same inputs as the
// B200 engine. Nothing in the product links or loads it.
//
// Every entry point takes host buffers, returns 0 on success and a negative
// code on a CUDA error, and runs synchronously on the legacy default stream
// exactly as the reference drivers do (main_stereo_hbp_isp.cu:31-76).
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <unistd.h>
#include <vector>

#include "hbp_isp.hpp"
#include "post_process.hpp"
#include "segment.hpp"
#include "stereo_cost.hpp"

// Kernels defined in the reference sources (external linkage); launched here
// one by one to pin individual stages.
__global__ void img_BGR_to_grey(const uchar3 *, float *, const int, const int);
__global__ void img_float1_to_uchar1(const float *, uint8_t *, const int, const int);
__global__ void img_uchar3_to_float4(const uchar3 *, float4 *, const int, const int);
__global__ void img_BGR_to_LAB(float4 *, const int, const int);
void img_gauss_blur(float4 *&, float4 *&, float *const, const double, const int, const int);
__global__ void compute_1nn_grid_k(const float4 *, int *, int2 *, float *, float *, const int,
                                   const int, const int);

namespace
{
int last_error()
{
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess)
        return -(int)e;
    e = cudaGetLastError();
    return e == cudaSuccess ? 0 : -(int)e;
}

cv::Mat wrap_bgr(const uint8_t *bgr, int W, int H)
{
    cv::Mat m(H, W, CV_8UC3);
    std::memcpy(m.data, bgr, (size_t)W * H * 3);
    return m;
}

// Exposes StereoCost's protected device buffers (stereo_cost.hpp:53-72).
struct StereoCostView : public StereoCost
{
    using StereoCost::StereoCost;
    const uint32_t *censusL() const { return imgL_trans_d; }
    const uint32_t *censusR() const { return imgR_trans_d; }
    const uint8_t *cost_u8() const { return img_cost_u1_d; }
    const uint8_t *greyL() const { return imgL_u1_d; }
    const uint8_t *greyR() const { return imgR_u1_d; }
    const float *greyL_f() const { return imgL_f1_d; }
    const float *greyR_f() const { return imgR_f1_d; }
};

__global__ void ref_patch_weight_k(float *out, float omega)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < 766)
    {
        float absdiff = (float)k;
        out[k] = expf(-absdiff / omega);
    }
}

template <typename T>
void d2h(T *dst, const T *src, size_t n)
{
    if (dst)
        cudaMemcpy(dst, src, sizeof(T) * n, cudaMemcpyDeviceToHost);
}
} // namespace

extern "C" {

// Grey conversion and u8 truncation (imutil.cu:116-130, :154-168).
int ref_grey(const uint8_t *bgr, int W, int H, float *grey_f, uint8_t *grey_u8)
{
    size_t n = (size_t)W * H;
    uchar3 *in_d;
    float *f_d;
    uint8_t *u_d;
    cudaMalloc(&in_d, n * 3);
    cudaMalloc(&f_d, n * 4);
    cudaMalloc(&u_d, n);
    cudaMemcpy(in_d, bgr, n * 3, cudaMemcpyHostToDevice);
    dim3 blk(32, 2), grd((W + 31) / 32, (H + 1) / 2);
    img_BGR_to_grey<<<grd, blk>>>(in_d, f_d, W, H);
    img_float1_to_uchar1<<<grd, blk>>>(f_d, u_d, W, H);
    int rc = last_error();
    d2h(grey_f, f_d, n);
    d2h(grey_u8, u_d, n);
    cudaFree(in_d);
    cudaFree(f_d);
    cudaFree(u_d);
    return rc;
}

// BGR u8 -> CIELAB float4 (L, a, b, 1) as SegHAC::img_CPU_to_GPU does with
// sigma = 0 (segment.cu:795-809).
int ref_lab(const uint8_t *bgr, int W, int H, float *lab4)
{
    size_t n = (size_t)W * H;
    uchar3 *in_d;
    float4 *f_d;
    cudaMalloc(&in_d, n * 3);
    cudaMalloc(&f_d, n * 16);
    cudaMemcpy(in_d, bgr, n * 3, cudaMemcpyHostToDevice);
    dim3 blk(32, 2), grd((W + 31) / 32, (H + 1) / 2);
    img_uchar3_to_float4<<<grd, blk>>>(in_d, f_d, W, H);
    img_BGR_to_LAB<<<grd, blk>>>(f_d, W, H);
    int rc = last_error();
    d2h(lab4, (const float *)f_d, n * 4);
    cudaFree(in_d);
    cudaFree(f_d);
    return rc;
}

// SegHAC::img_CPU_to_GPU (segment.cu:795-809) with sigma: the float4 BGR
// image, the Gaussian blur img_gauss_blur (imutil.cu:397-497) when
// sigma > FLT_MIN, then BGR -> LAB.
int ref_lab_sigma(const uint8_t *bgr, int W, int H, double sigma, float *lab4)
{
    size_t n = (size_t)W * H;
    uchar3 *in_d;
    float4 *f_d, *buf_d;
    float *filter_d;
    cudaMalloc(&in_d, n * 3);
    cudaMalloc(&f_d, n * 16);
    cudaMalloc(&buf_d, n * 16);
    cudaMalloc(&filter_d, sizeof(float) * 64 * 64);
    cudaMemcpy(in_d, bgr, n * 3, cudaMemcpyHostToDevice);
    dim3 blk(32, 2), grd((W + 31) / 32, (H + 1) / 2);
    img_uchar3_to_float4<<<grd, blk>>>(in_d, f_d, W, H);
    float4 *img = f_d, *buf = buf_d;
    if (sigma > FLT_MIN)
        img_gauss_blur(img, buf, filter_d, sigma, W, H);
    img_BGR_to_LAB<<<grd, blk>>>(img, W, H);
    int rc = last_error();
    d2h(lab4, (const float *)img, n * 4);
    cudaFree(in_d);
    cudaFree(f_d);
    cudaFree(buf_d);
    cudaFree(filter_d);
    return rc;
}

// SegHAC(link, num_nb, sigma, LabelISPFormat, target).run_ms() (segment.cu:
// 1279-1321; target > 1: the superpixel mode, get_target_clus :1016-1041),
// outputs as ref_segment (bd capacity 2 * num_nb * HW pairs, bdl
// num_nb * 2 * HW). Returns the number of levels.
int ref_segment_target(const uint8_t *bgr, int W, int H, int link, int num_nb, double sigma, int target,
                       int max_levels, int *level_sizes, int *clus, float *mean, int *bd, int *bdl)
{
    int levels = 0;
    int rc;
    {
        SegHAC seg(wrap_bgr(bgr, W, H), (Linkage)link, num_nb, sigma, LabelISPFormat, target, false);
        seg.run_ms();
        rc = last_error();
        std::vector<int> nc = seg.g_num_clus_isp(), nb = seg.g_num_bd_isp();
        levels = (int)nc.size();
        size_t tc = 0, tb = 0;
        for (int i = 0; i < levels; ++i)
        {
            if (i < max_levels)
            {
                level_sizes[2 * i] = nc[i];
                level_sizes[2 * i + 1] = nb[i];
            }
            tc += nc[i];
            tb += nb[i];
        }
        d2h(clus, seg.g_isp_clus_d(), tc);
        d2h(mean, seg.g_isp_mean_d(), tc * 6);
        d2h(bd, (const int *)seg.g_isp_bd_d(), tb * 2);
        d2h(bdl, seg.g_isp_bdl_d(), tb);
    }
    int rc2 = last_error();
    if (rc || rc2)
        return rc ? rc : rc2;
    return levels;
}

// The same with target 1 (the pyramid up to one node).
int ref_segment_cfg(const uint8_t *bgr, int W, int H, int link, int num_nb, double sigma, int max_levels,
                    int *level_sizes, int *clus, float *mean, int *bd, int *bdl)
{
    return ref_segment_target(bgr, W, H, link, num_nb, sigma, 1, max_levels, level_sizes, clus, mean, bd, bdl);
}

// Pixel 1-NN on the 4-grid (segment.cu:57-195): nn, dist_min and the four
// directed distances per pixel (dist4[4*i+k], k = up, down, left, right; the
// entry is left untouched where the neighbour does not exist).
int ref_1nn_grid(const float *lab4, int W, int H, int *nn, float *dist_min, float *dist4)
{
    size_t n = (size_t)W * H;
    float4 *img_d;
    int *nn_d;
    int2 *bd_d;
    float *dist_d, *dmin_d;
    cudaMalloc(&img_d, n * 16);
    cudaMalloc(&nn_d, n * 4);
    cudaMalloc(&bd_d, n * 4 * 8);
    cudaMalloc(&dist_d, n * 4 * 4);
    cudaMalloc(&dmin_d, n * 4);
    cudaMemcpy(img_d, lab4, n * 16, cudaMemcpyHostToDevice);
    dim3 blk(32, 2), grd((W + 31) / 32, (H + 1) / 2);
    compute_1nn_grid_k<<<grd, blk>>>(img_d, nn_d, bd_d, dist_d, dmin_d, 4, W, H);
    int rc = last_error();
    d2h(nn, nn_d, n);
    d2h(dist_min, dmin_d, n);
    d2h(dist4, dist_d, n * 4);
    cudaFree(img_d);
    cudaFree(nn_d);
    cudaFree(bd_d);
    cudaFree(dist_d);
    cudaFree(dmin_d);
    return rc;
}

// CRTrees::get_clus + compact_clus_label (CRTrees.cu:395-434, :467-483) on a
// host successor array. Returns the number of clusters (>= 0) or an error.
int ref_crtrees(const int *nn, int N, int *clus)
{
    int *nn_d, *clus_d;
    cudaMalloc(&nn_d, sizeof(int) * N);
    cudaMalloc(&clus_d, sizeof(int) * N);
    cudaMemcpy(nn_d, nn, sizeof(int) * N, cudaMemcpyHostToDevice);
    int num = 0;
    {
        CRTrees tr(N);
        tr.get_clus(nn_d, clus_d, N);
        num = tr.compact_clus_label(clus_d, N);
    }
    int rc = last_error();
    d2h(clus, clus_d, N);
    cudaFree(nn_d);
    cudaFree(clus_d);
    return rc ? rc : num;
}

// Census/Hamming/WTA through StereoCost (stereo_cost.cu:421-445). Outputs
// (each optional): both census images, the u8 volume [HW][D_align], the float
// volume [D][HW], the WTA disparity; with to_right != 0 the float volume and
// WTA are those after cost_to_right() (stereo_cost.cu:488-516).
int ref_cost(const uint8_t *bgrL, const uint8_t *bgrR, int W, int H, int D, int to_right,
             uint8_t *greyL, uint8_t *greyR, uint32_t *censusL, uint32_t *censusR,
             uint8_t *vol_u8, float *vol_f32, float *wta)
{
    size_t n = (size_t)W * H;
    int Da = (D + 31) / 32 * 32;
    int rc;
    {
        StereoCostView sc(wrap_bgr(bgrL, W, H), wrap_bgr(bgrR, W, H), D, "");
        sc.compute_stereo_cost("Census");
        if (to_right)
            sc.cost_to_right();
        rc = last_error();
        d2h(greyL, sc.greyL(), n);
        d2h(greyR, sc.greyR(), n);
        d2h(censusL, sc.censusL(), n);
        d2h(censusR, sc.censusR(), n);
        d2h(vol_u8, sc.cost_u8(), n * Da);
        d2h(vol_f32, sc.g_img_cost_d(), n * D);
        d2h(wta, sc.g_img_D_d(), n);
    }
    int rc2 = last_error();
    return rc ? rc : rc2;
}

// SegHAC(CentroidLink, 4-grid, sigma 0, LabelISPFormat, target 1).run_ms()
// (segment.cu:1279-1321). level_sizes receives, per pushed ISP level,
// (num_clus, num_bd). clus/mean/bd/bdl receive the concatenated ISP arrays
// (capacity 2*HW, 12*HW, 16*HW ints, 8*HW). Returns the number of levels.
int ref_segment(const uint8_t *bgr, int W, int H, int max_levels, int *level_sizes, int *clus,
                float *mean, int *bd, int *bdl)
{
    int levels = 0;
    int rc;
    {
        SegHAC seg(wrap_bgr(bgr, W, H), CentoridLink, 4, 0.0, LabelISPFormat, 1, false);
        seg.run_ms();
        rc = last_error();
        std::vector<int> nc = seg.g_num_clus_isp(), nb = seg.g_num_bd_isp();
        levels = (int)nc.size();
        size_t tc = 0, tb = 0;
        for (int i = 0; i < levels; ++i)
        {
            if (i < max_levels)
            {
                level_sizes[2 * i] = nc[i];
                level_sizes[2 * i + 1] = nb[i];
            }
            tc += nc[i];
            tb += nb[i];
        }
        d2h(clus, seg.g_isp_clus_d(), tc);
        d2h(mean, seg.g_isp_mean_d(), tc * 6);
        d2h(bd, (const int *)seg.g_isp_bd_d(), tb * 2);
        d2h(bdl, seg.g_isp_bdl_d(), tb);
    }
    int rc2 = last_error();
    if (rc || rc2)
        return rc ? rc : rc2;
    return levels;
}

// The single-pair driver path (main_stereo_hbp_isp.cu:33-72): SegHAC on the
// left image, Census cost, HBP_ISP(alpha, tau_smooth).run_ms(min_level).
// With right_view != 0 it runs the right-view path of main_bench_middv3.cu:
// 189-203 instead (SegHAC on the right image, cost_to_right). Outputs the
// disparity (HW floats) and plane labels (HW x 3 floats). Returns the number
// of ISP levels.
int ref_hbp_pair(const uint8_t *bgrL, const uint8_t *bgrR, int W, int H, int D, float alpha,
                 float tau_smooth, int min_level, int right_view, float *disp, float *plane)
{
    int levels = 0;
    int rc;
    {
        cv::Mat L = wrap_bgr(bgrL, W, H), R = wrap_bgr(bgrR, W, H);
        SegHAC *seg = new SegHAC(right_view ? R : L, CentoridLink, 4, 0.0, LabelISPFormat, 1, false);
        seg->run_ms();
        ISPData *isp = new ISPData(seg);
        levels = (int)seg->g_num_clus_isp().size();
        delete seg;
        StereoCost *sc = new StereoCost(L, R, D, "");
        sc->compute_stereo_cost("Census");
        if (right_view)
            sc->cost_to_right();
        StereoData *sd = new StereoData(sc, true);
        delete sc;
        HBP_ISP *hbp = new HBP_ISP(isp, sd, alpha, tau_smooth);
        std::pair<cv::Mat, cv::Mat> res = hbp->run_ms(min_level);
        rc = last_error();
        std::memcpy(disp, res.first.data, sizeof(float) * (size_t)W * H);
        std::memcpy(plane, res.second.data, sizeof(float) * (size_t)W * H * 3);
        delete hbp;
        delete sd;
        delete isp;
    }
    int rc2 = last_error();
    if (rc || rc2)
        return rc ? rc : rc2;
    return levels;
}

// PostProcess::left_right_check + plane_label_to_disp (post_process.cu:47-110,
// :373-390) and, with do_median == 1, median_filter + plane_label_to_disp
// (:127-185, CPU); with do_median == 2, median_filter_gpu (:245-371) instead.
// dispL/planeL are updated in place; dispR/planeR are read.
int ref_post(const uint8_t *bgrL, const uint8_t *bgrR, int W, int H, float *dispL, float *planeL,
             float *dispR, float *planeR, int do_median)
{
    cv::Mat L = wrap_bgr(bgrL, W, H), R = wrap_bgr(bgrR, W, H);
    std::pair<cv::Mat, cv::Mat> left(cv::Mat(H, W, CV_32FC1), cv::Mat(H, W, CV_32FC3));
    std::pair<cv::Mat, cv::Mat> right(cv::Mat(H, W, CV_32FC1), cv::Mat(H, W, CV_32FC3));
    size_t n = (size_t)W * H;
    std::memcpy(left.first.data, dispL, n * 4);
    std::memcpy(left.second.data, planeL, n * 12);
    std::memcpy(right.first.data, dispR, n * 4);
    std::memcpy(right.second.data, planeR, n * 12);
    PostProcess pp(L, R);
    pp.left_right_check(left, right);
    pp.plane_label_to_disp(left, right);
    if (do_median == 2)
    {
        pp.median_filter_gpu(left, right);
        pp.plane_label_to_disp(left, right);
    }
    else if (do_median)
    {
        pp.median_filter(left, right);
        pp.plane_label_to_disp(left, right);
    }
    std::memcpy(dispL, left.first.data, n * 4);
    std::memcpy(planeL, left.second.data, n * 12);
    return 0;
}

// compute_patch_weight's expression (post_process.cu:199-213) for every
// colour distance k = 0..765 (the distance of two BGR8 pixels is an integer):
// expf(-k / 10.0f) on the device, as median_filter_gpu evaluates it.
int ref_patch_weights(float *out766)
{
    float *d;
    cudaMalloc(&d, sizeof(float) * 766);
    ref_patch_weight_k<<<(766 + 127) / 128, 128>>>(d, 10.0f);
    int rc = last_error();
    d2h(out766, d, 766);
    cudaFree(d);
    return rc;
}

// The MC-CNN single-view path (main_bench_middv3.cu:73-108 with cost
// "MC-CNN"): the float volume src [D][H][W] goes through the reference's own
// file reader (stereo_cost.cu:396-418: out-of-view fill, truncation at 0.5)
// from a raw temporary file, then WTA, SegHAC on the left image and
// HBP_ISP(alpha, tau_smooth).run_ms(min_level). With right_view != 0, the
// right view of main_bench_middv3.cu:189-203 instead (SegHAC on the right
// image, cost_to_right). vol_f32 ([D][HW]) and wta receive the stored volume
// and WTA (optional). Returns the number of levels.
static double g_last_hbp_ms = 0.0;

// Milliseconds of the last ref_hbp_f32's HBP_ISP construction + run_ms, the
// scope main_bench_middv3.cu:97-104 times.
double ref_last_hbp_ms() { return g_last_hbp_ms; }

int ref_hbp_f32(const uint8_t *bgrL, const uint8_t *bgrR, const float *src, int W, int H, int D,
                float alpha, float tau_smooth, int min_level, int right_view, float *vol_f32, float *wta,
                float *disp, float *plane)
{
    char path[] = "/tmp/hbpref_volXXXXXX";
    int fd = mkstemp(path);
    if (fd < 0)
        return -1000;
    size_t n = (size_t)W * H, bytes = n * D * sizeof(float);
    bool ok = write(fd, src, bytes) == (ssize_t)bytes;
    close(fd);
    if (!ok)
    {
        unlink(path);
        return -1001;
    }
    int levels = 0;
    int rc;
    {
        cv::Mat L = wrap_bgr(bgrL, W, H), R = wrap_bgr(bgrR, W, H);
        SegHAC *seg = new SegHAC(right_view ? R : L, CentoridLink, 4, 0.0, LabelISPFormat, 1, false);
        seg->run_ms();
        ISPData *isp = new ISPData(seg);
        levels = (int)seg->g_num_clus_isp().size();
        delete seg;
        StereoCost *sc = new StereoCost(L, R, D, std::string(path));
        sc->compute_stereo_cost("MC-CNN");
        if (right_view)
            sc->cost_to_right();
        d2h(vol_f32, sc->g_img_cost_d(), n * D);
        d2h(wta, sc->g_img_D_d(), n);
        StereoData *sd = new StereoData(sc, true);
        delete sc;
        cudaDeviceSynchronize();
        auto c0 = std::chrono::steady_clock::now();
        HBP_ISP *hbp = new HBP_ISP(isp, sd, alpha, tau_smooth);
        std::pair<cv::Mat, cv::Mat> res = hbp->run_ms(min_level);
        auto c1 = std::chrono::steady_clock::now();
        g_last_hbp_ms = std::chrono::duration<double, std::milli>(c1 - c0).count();
        rc = last_error();
        std::memcpy(disp, res.first.data, sizeof(float) * n);
        std::memcpy(plane, res.second.data, sizeof(float) * n * 3);
        delete hbp;
        delete sd;
        delete isp;
    }
    unlink(path);
    int rc2 = last_error();
    if (rc || rc2)
        return rc ? rc : rc2;
    return levels;
}

// The AD cost path: StereoCost::compute_stereo_cost("AD") (stereo_cost.cu:
// 421-429), optionally cost_to_right, then SegHAC on the view's image and
// HBP_ISP(alpha, tau_smooth).run_ms(min_level) as ref_hbp_pair. greyL/greyR
// (float HW), vol_f32 ([D][HW]) and wta are optional outputs. Returns the
// number of levels.
int ref_hbp_ad(const uint8_t *bgrL, const uint8_t *bgrR, int W, int H, int D, float alpha, float tau_smooth,
               int min_level, int right_view, float *greyL, float *greyR, float *vol_f32, float *wta, float *disp,
               float *plane)
{
    size_t n = (size_t)W * H;
    int levels = 0;
    int rc;
    {
        cv::Mat L = wrap_bgr(bgrL, W, H), R = wrap_bgr(bgrR, W, H);
        SegHAC *seg = new SegHAC(right_view ? R : L, CentoridLink, 4, 0.0, LabelISPFormat, 1, false);
        seg->run_ms();
        ISPData *isp = new ISPData(seg);
        levels = (int)seg->g_num_clus_isp().size();
        delete seg;
        StereoCostView *sc = new StereoCostView(L, R, D, "");
        sc->compute_stereo_cost("AD");
        if (right_view)
            sc->cost_to_right();
        d2h(greyL, sc->greyL_f(), n);
        d2h(greyR, sc->greyR_f(), n);
        d2h(vol_f32, sc->g_img_cost_d(), n * D);
        d2h(wta, sc->g_img_D_d(), n);
        StereoData *sd = new StereoData(sc, true);
        delete sc;
        HBP_ISP *hbp = new HBP_ISP(isp, sd, alpha, tau_smooth);
        std::pair<cv::Mat, cv::Mat> res = hbp->run_ms(min_level);
        rc = last_error();
        std::memcpy(disp, res.first.data, sizeof(float) * n);
        std::memcpy(plane, res.second.data, sizeof(float) * n * 3);
        delete hbp;
        delete sd;
        delete isp;
    }
    int rc2 = last_error();
    if (rc || rc2)
        return rc ? rc : rc2;
    return levels;
}

} // extern "C"
