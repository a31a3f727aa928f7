// Round trip of the PFM reader/writer and the evaluator of include/hbp_isp/io.hpp.
// usage: io_check dir W H   (dir holds disp.f32, gt.f32, nonocc.u8 and py.pfm)
// Writes dir/cpp1.pfm, dir/cpp3.pfm and prints "all nonocc occ" for threshold
// 1.0 and 2.0, then the first value of py.pfm's top-left pixel.
#include <cstdio>
#include <cstdlib>
#include <fstream>

#include "hbp_isp/io.hpp"

using hbp_isp::Mat;

static Mat load(const std::string &path, int W, int H, int type)
{
    Mat m(H, W, type);
    std::ifstream f(path, std::ios::binary);
    f.read(reinterpret_cast<char *>(m.data), (std::streamsize)m.bytes());
    return m;
}

int main(int argc, char **argv)
{
    if (argc != 4)
        return 2;
    const std::string dir = argv[1];
    const int W = std::atoi(argv[2]), H = std::atoi(argv[3]);
    Mat disp = load(dir + "/disp.f32", W, H, hbp_isp::MAT_32FC1);
    Mat gt = load(dir + "/gt.f32", W, H, hbp_isp::MAT_32FC1);
    Mat mask = load(dir + "/nonocc.u8", W, H, hbp_isp::MAT_8UC1);
    // 1 and 3 channels through the writer and back
    Mat three(H, W, hbp_isp::MAT_32FC3);
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < 3 * W; ++x)
            three.ptr<float>(y)[x] = disp.ptr<float>(y)[x / 3] + (float)(x % 3);
    if (!cvutils::io::save_pfm_file(dir + "/cpp1.pfm", disp) || !cvutils::io::save_pfm_file(dir + "/cpp3.pfm", three))
        return 3;
    Mat r1 = cvutils::io::read_pfm_file(dir + "/cpp1.pfm"), r3 = cvutils::io::read_pfm_file(dir + "/cpp3.pfm");
    if (r1.empty() || r3.empty() || std::memcmp(r1.data, disp.data, disp.bytes()) ||
        std::memcmp(r3.data, three.data, three.bytes()))
        return 4;
    Evaluator ev(gt, mask);
    for (double t : {1.0, 2.0})
    {
        ev.setErrorThreshold(t);
        const auto r = ev.evaluate(disp);
        std::printf("%.10f %.10f %.10f\n", r.all, r.nonocc, r.occ);
    }
    Mat py = cvutils::io::read_pfm_file(dir + "/py.pfm");
    if (py.empty())
        return 5;
    std::printf("%.6f\n", py.ptr<float>(0)[0]);
    return 0;
}
