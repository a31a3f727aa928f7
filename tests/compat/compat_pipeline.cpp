// The reference's two driver flows written against the reference-interface
// classes of include/hbp_isp/:
//   single: main_stereo_hbp_isp.cu:33-76 (SegHAC -> ISPData, StereoCost ->
//           StereoData, HBP_ISP::run_ms, medianFilter)
//   lr:     main_bench_middv3.cu:169-219 (both views, LR check, fill,
//           weighted median, plane -> disparity)
// with the Census and AD costs (alpha 1000.1) and, given an im0.acrt-style
// volume file, the MC-CNN cost (alpha 1.3, bench_MiddV3_train.sh:6). Writes
// <out_prefix>{census,ad,mccnn}_{single,lr,lr_gpu,levels}.f32 (lr_gpu: the LR
// flow with median_filter_gpu; levels: every level's disparity from
// HBP_ISP::run_ms_vis, top level first), and SegHAC's pictures of the left
// image (segment.cu:1096-1111): <out_prefix>seg_{int,u3,bd}_t{1,60}.bin, the
// pictures of run_ms(&segs) concatenated.
// usage: compat_pipeline left.bgr right.bgr W H D out_prefix [vol.acrt]
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <tuple>

#include "hbp_isp/hbp_isp_all.hpp"

using hbp_isp::Mat;

static Mat read_bgr(const char *path, int W, int H)
{
    Mat m(H, W, hbp_isp::MAT_8UC3);
    std::ifstream f(path, std::ios::binary);
    f.read(reinterpret_cast<char *>(m.data), (std::streamsize)m.bytes());
    if (!f)
        throw std::runtime_error(std::string("cannot read ") + path);
    return m;
}

static void write_f32(const char *path, const Mat &m)
{
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char *>(m.data), (std::streamsize)m.bytes());
}

static void flows(const Mat &L, const Mat &R, int D, const std::string &cost, const std::string &vol_dir,
                  float alpha, const std::string &out)
{
    const float tau_smooth = 0.6f;
    const int min_level = 2;

    // single-pair driver
    SegHAC *seg = new SegHAC(L, CentoridLink, 4, 0, LabelISPFormat, 1, false);
    seg->run_ms();
    ISPData *isp = new ISPData(seg);
    delete seg;
    StereoCost *sc = new StereoCost(L, R, D, vol_dir);
    sc->compute_stereo_cost(cost);
    StereoData *sd = new StereoData(sc, true);
    delete sc;
    HBP_ISP *hbp = new HBP_ISP(isp, sd, alpha, tau_smooth);
    auto results_left = hbp->run_ms(min_level);
    Mat disp = results_left.first.clone();
    medianFilter(disp);
    write_f32((out + "_single.f32").c_str(), disp);
    {
        // every level's map (run_ms_vis), top level first, concatenated
        std::ofstream f(out + "_levels.f32", std::ios::binary);
        for (const auto &lv : hbp->run_ms_vis(min_level))
            f.write(reinterpret_cast<const char *>(std::get<0>(lv).data), (std::streamsize)std::get<0>(lv).bytes());
    }

    // MidV3_LR: the right view, then LR check, fill and weighted median
    SegHAC *seg_r = new SegHAC(R, CentoridLink, 4, 0, LabelISPFormat, 1, false);
    seg_r->run_ms();
    ISPData *isp_r = new ISPData(seg_r);
    delete seg_r;
    StereoCost *sc_r = new StereoCost(L, R, D, vol_dir);
    sc_r->compute_stereo_cost(cost);
    sc_r->cost_to_right();
    StereoData *sd_r = new StereoData(sc_r, true);
    delete sc_r;
    HBP_ISP *hbp_r = new HBP_ISP(isp_r, sd_r, alpha, tau_smooth);
    auto results_right = hbp_r->run_ms(min_level);
    PostProcess *post = new PostProcess(L, R);
    post->left_right_check(results_left, results_right);
    post->plane_label_to_disp(results_left, results_right);
    // the reference's GPU variant of the weighted median, on a copy
    std::pair<Mat, Mat> gpu_left(results_left.first.clone(), results_left.second.clone());
    post->median_filter_gpu(gpu_left, results_right);
    post->plane_label_to_disp(gpu_left, results_right);
    write_f32((out + "_lr_gpu.f32").c_str(), gpu_left.first);
    post->median_filter(results_left, results_right);
    post->plane_label_to_disp(results_left, results_right);
    write_f32((out + "_lr.f32").c_str(), results_left.first);

    delete post;
    delete hbp_r;
    delete sd_r;
    delete isp_r;
    delete hbp;
    delete sd;
    delete isp;
}

// SegHAC on a stream (segment.hpp:87-107): after set_frame / set_seq_img and
// run_ms, the pyramid equals a fresh SegHAC's on the same image, and the
// device getters point at it.
static void stream_check(const Mat &L, const Mat &R)
{
    auto isp_of = [](SegHAC &s) {
        ISPData isp(&s);
        std::vector<int> clus, bd, bdl;
        std::vector<float> mean;
        isp.copy_isp(clus, mean, bd, bdl);
        if (!isp.g_isp_clus_d() || !isp.g_isp_mean_d() || !isp.g_isp_bd_d() || !isp.g_isp_bdl_d())
            throw std::runtime_error("ISPData device getters returned null");
        return std::make_tuple(clus, mean, bd, bdl, isp.g_num_clus_isp());
    };
    SegHAC video(L, CentoridLink, 4, 0, LabelISPFormat, 1, false);
    video.run_ms();
    video.set_frame(R);
    video.run_ms();
    SegHAC fresh(R, CentoridLink, 4, 0, LabelISPFormat, 1, false);
    fresh.run_ms();
    if (isp_of(video) != isp_of(fresh) || video.g_num_clus_isp() != fresh.g_num_clus_isp())
        throw std::runtime_error("set_frame + run_ms differs from a fresh SegHAC");
    video.set_seq_img(L);
    video.run_ms();
    SegHAC fresh_l(L, CentoridLink, 4, 0, LabelISPFormat, 1, false);
    fresh_l.run_ms();
    if (isp_of(video) != isp_of(fresh_l))
        throw std::runtime_error("set_seq_img + run_ms differs from a fresh SegHAC");
}

// SegHAC's picture formats: the full hierarchy (target 1, one picture per
// level) and 60 superpixels (one picture), Ward linkage with 8 neighbours.
static void seg_pictures(const Mat &L, const std::string &out)
{
    const std::pair<SegFormat, const char *> fmts[] = {
        {LabelIntFormat, "int"}, {LabelUchar3Format, "u3"}, {BoundaryFormat, "bd"}};
    for (int target : {1, 60})
        for (const auto &f : fmts)
        {
            SegHAC seg(L, WardLink, 8, 0, f.first, target, false);
            std::vector<Mat> segs;
            seg.run_ms(&segs);
            if ((int)segs.size() != (target == 1 ? seg.g_levels() : 1))
                throw std::runtime_error("SegHAC::run_ms gave the wrong number of pictures");
            std::ofstream o(out + "seg_" + f.second + "_t" + std::to_string(target) + ".bin", std::ios::binary);
            for (const Mat &m : segs)
                o.write(reinterpret_cast<const char *>(m.data), (std::streamsize)m.bytes());
        }
    // the formats that give no picture
    std::vector<Mat> segs;
    SegHAC dev(L, WardLink, 8, 0, LabelDeviceIntFormat, 1, false);
    dev.run_ms(&segs);
    for (const Mat &m : segs)
        if (!m.empty())
            throw std::runtime_error("LabelDeviceIntFormat gave a picture");
    if ((int)segs.size() != dev.g_levels())
        throw std::runtime_error("LabelDeviceIntFormat: one empty picture per level expected");
    SegHAC none(L, WardLink, 8, 0, EmptyFormat, 1, false);
    segs.clear();
    none.run_ms(&segs);
    if (!segs.empty())
        throw std::runtime_error("EmptyFormat gave pictures");
}

int main(int argc, char **argv)
{
    if (argc != 7 && argc != 8)
    {
        std::fprintf(stderr, "usage: %s left.bgr right.bgr W H D out_prefix [vol.acrt]\n", argv[0]);
        return 2;
    }
    const int W = std::atoi(argv[3]), H = std::atoi(argv[4]), D = std::atoi(argv[5]);
    const std::string out(argv[6]);
    try
    {
        Mat L = read_bgr(argv[1], W, H), R = read_bgr(argv[2], W, H);
        stream_check(L, R);
        seg_pictures(L, out);
        flows(L, R, D, "Census", "", 1000.1f, out + "census");
        flows(L, R, D, "AD", "", 1000.1f, out + "ad");
        if (argc == 8)
            flows(L, R, D, "MC-CNN", argv[7], 1.3f, out + "mccnn");
    }
    catch (const std::exception &e)
    {
        std::fprintf(stderr, "compat_pipeline: %s\n", e.what());
        return 1;
    }
    return 0;
}
